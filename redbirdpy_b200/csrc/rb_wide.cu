// Wide-field (pattern) sources and detectors: dense right-hand-side columns
// that redbirdpy keeps in cfg['widesrc'] / cfg['widedet'] (Nn x Npattern, from
// src2bc or the caller), placed in the RHS after the point columns of their
// kind (column order [point src | wide src | point det | wide det],
// redbirdpy/forward.py:278-352), and the detector readout of the wide
// detectors, rhs_det^T phi_src over all nodes (forward.py:430-442).
#include <algorithm>

#include "rb_common.cuh"

namespace rb {

// B[n][col0 + j] = W[n][j] for the w pattern columns
__global__ void wide_rhs_kernel(const double* __restrict__ W, int64_t nn, int64_t w, int64_t ldw, int64_t ld,
                                int64_t col0, double* __restrict__ B) {
  const int64_t total = nn * w;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t n = t / w, j = t - n * w;
    B[n * ld + col0 + j] = W[n * ldw + j];
  }
}

// Partial sums over a slab of nodes of detval[d][s] = sum_n W[n][d] phi[n][s]:
// block b takes nodes [b * rows, (b + 1) * rows), thread t the (d, s) pairs
// t, t + blockDim, ...; the slabs are added in a second pass in slab order,
// so the result is the same on every run.
template <typename T>
__global__ void wide_det_part_kernel(const double* __restrict__ W, int64_t nn, int64_t wd, int64_t ldw,
                                     const T* __restrict__ phi, int64_t ld, int64_t nsrc, int64_t rows,
                                     T* __restrict__ part) {
  const int64_t n0 = blockIdx.x * rows, n1 = std::min<int64_t>(nn, n0 + rows);
  const int64_t npair = wd * nsrc;
  for (int64_t p = threadIdx.x; p < npair; p += blockDim.x) {
    const int64_t d = p / nsrc, s = p - d * nsrc;
    T acc = s_zero(T());
    for (int64_t n = n0; n < n1; ++n) {
      T wv = s_zero(T());
      if constexpr (Scalar<T>::is_complex) wv.x = W[n * ldw + d];
      else wv = W[n * ldw + d];
      acc = s_fma(wv, phi[n * ld + s], acc);
    }
    part[blockIdx.x * npair + p] = acc;
  }
}

template <typename T>
__global__ void wide_det_sum_kernel(const T* __restrict__ part, int64_t slabs, int64_t npair, T* __restrict__ out) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= npair) return;
  T acc = s_zero(T());
  for (int64_t b = 0; b < slabs; ++b) acc = s_add(acc, part[b * npair + p]);
  out[p] = acc;
}

constexpr int64_t kWideSlabs = 512;

}  // namespace rb

using namespace rb;

extern "C" {

int rb_wide_rhs(const double* W, int64_t nn, int64_t w, int64_t ldw, int64_t ld, int64_t col0, double* B,
                void* stream) {
  if (!W || !B || nn < 1 || w < 0 || ldw < w || col0 < 0 || col0 + w > ld)
    return fail(RB_EARG, "rb_wide_rhs: bad arguments");
  if (w == 0) return RB_OK;
  const unsigned g = (unsigned)std::min<int64_t>(ceil_div(nn * w, 256), 148 * 32);
  wide_rhs_kernel<<<g, 256, 0, as_stream(stream)>>>(W, nn, w, ldw, ld, col0, B);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

size_t rb_wide_getdet_work_bytes(int64_t wd, int64_t nsrc, int32_t kind) {
  return (size_t)kWideSlabs * wd * nsrc * (kind == RB_C128 ? 16 : 8) + 256;
}

int rb_wide_getdet(const double* W, int64_t nn, int64_t wd, int64_t ldw, const void* phi, int64_t ld, int64_t nsrc,
                   int32_t kind, void* detval, void* work, size_t work_bytes, void* stream) {
  if (!W || !phi || !detval || nn < 1 || wd < 0 || ldw < wd || nsrc < 0 || nsrc > ld)
    return fail(RB_EARG, "rb_wide_getdet: bad arguments");
  if (kind != RB_F64 && kind != RB_C128) return fail(RB_EARG, "rb_wide_getdet: kind must be RB_F64 or RB_C128");
  const int64_t npair = wd * nsrc;
  if (npair == 0) return RB_OK;
  if (!work || work_bytes < rb_wide_getdet_work_bytes(wd, nsrc, kind))
    return fail(RB_EARG, "rb_wide_getdet: workspace too small");
  const int64_t slabs = std::min<int64_t>(kWideSlabs, nn);
  const int64_t rows = ceil_div(nn, slabs);
  const int64_t used = ceil_div(nn, rows);
  cudaStream_t st = as_stream(stream);
  if (kind == RB_F64) {
    wide_det_part_kernel<double><<<(unsigned)used, 256, 0, st>>>(W, nn, wd, ldw, (const double*)phi, ld, nsrc, rows,
                                                                  (double*)work);
    RB_LAUNCH_CHECK();
    wide_det_sum_kernel<double><<<(unsigned)ceil_div(npair, 256), 256, 0, st>>>((const double*)work, used, npair,
                                                                                (double*)detval);
  } else {
    wide_det_part_kernel<cdouble><<<(unsigned)used, 256, 0, st>>>(W, nn, wd, ldw, (const cdouble*)phi, ld, nsrc,
                                                                   rows, (cdouble*)work);
    RB_LAUNCH_CHECK();
    wide_det_sum_kernel<cdouble><<<(unsigned)ceil_div(npair, 256), 256, 0, st>>>((const cdouble*)work, used, npair,
                                                                                 (cdouble*)detval);
  }
  RB_LAUNCH_CHECK();
  return RB_OK;
}

}  // extern "C"
