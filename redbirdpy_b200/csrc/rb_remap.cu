// Gauss-Newton matrix assembly across wavelengths, chromophores and meshes:
//   rb_jac_remap   dual-mesh reconstruction (redbirdpy/recon.py:818-876): the
//                  Jacobian columns of the forward mesh's nodes distributed to
//                  the reconstruction mesh's nodes by the barycentric weights
//                  of the recon element holding each forward node,
//                  out[r][q] = sum_{(i, w) in map(q)} w J[r][i], the map's
//                  entries of each q in ascending forward node order (the
//                  reference's accumulation order);
//   rb_jac_block   one wavelength's rows scaled into a block of the stacked
//                  real matrix (jacchrome's extinction weights,
//                  forward.py:572-589, and matreform's 'real', 'reim' and
//                  'logphase' forms of complex rows, recon.py:512-567).
#include <algorithm>

#include "rb_common.cuh"

namespace rb {

// one warp per (row, chunk of 32 output columns): lanes own output columns
template <typename T>
__global__ void jac_remap_kernel(const T* __restrict__ J, int64_t rows, int64_t ldj, const int32_t* __restrict__ mptr,
                                 const int32_t* __restrict__ midx, const double* __restrict__ mw, int64_t nq,
                                 T* __restrict__ out, int64_t ldo) {
  const int64_t total = rows * nq;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = t / nq, q = t - r * nq;
    const T* jr = J + r * ldj;
    T acc = s_zero(T());
    for (int32_t p = mptr[q]; p < mptr[q + 1]; ++p) {
      T w = s_zero(T());
      if constexpr (Scalar<T>::is_complex) w.x = (typename Scalar<T>::real)mw[p];
      else w = (T)mw[p];
      acc = s_fma(w, jr[midx[p]], acc);
    }
    out[r * ldo + q] = acc;
  }
}

// v = src[r][c] * (sre + i sim) * rowscale[r] (rowscale complex, optional);
// dst (FP32 rows, ldd) [row_re + r][col0 + c] = Re v and, when row_im >= 0,
// [row_im + r][col0 + c] = Im v
template <typename T>
__global__ void jac_block_kernel(const T* __restrict__ src, int64_t rows, int64_t cols, int64_t lds, double sre,
                                 double sim, const double* __restrict__ rowscale, float* __restrict__ dst, int64_t ldd,
                                 int64_t row_re, int64_t row_im, int64_t col0) {
  const int64_t total = rows * cols;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = t / cols, c = t - r * cols;
    const T v = src[r * lds + c];
    double a, b;
    if constexpr (Scalar<T>::is_complex) {
      a = v.x;
      b = v.y;
    } else {
      a = v;
      b = 0.0;
    }
    double fr = sre, fi = sim;
    if (rowscale) {
      const double gr = rowscale[2 * r], gi = rowscale[2 * r + 1];
      const double tr = fr * gr - fi * gi;
      fi = fr * gi + fi * gr;
      fr = tr;
    }
    dst[(row_re + r) * ldd + col0 + c] = (float)(a * fr - b * fi);
    if (row_im >= 0) dst[(row_im + r) * ldd + col0 + c] = (float)(a * fi + b * fr);
  }
}

}  // namespace rb

using namespace rb;

extern "C" {

int rb_jac_remap(const void* J, int32_t kind, int64_t rows, int64_t ldj, const int32_t* map_ptr,
                 const int32_t* map_idx, const double* map_w, int64_t nq, void* out, int64_t ldo, void* stream) {
  if (!J || !map_ptr || !out || rows < 0 || nq < 0 || ldo < nq) return fail(RB_EARG, "rb_jac_remap: bad arguments");
  if (rows * nq == 0) return RB_OK;
  const unsigned g = (unsigned)std::min<int64_t>(ceil_div(rows * nq, 256), 148 * 64);
  cudaStream_t st = as_stream(stream);
  switch (kind) {
    case RB_F32:
      jac_remap_kernel<float><<<g, 256, 0, st>>>((const float*)J, rows, ldj, map_ptr, map_idx, map_w, nq, (float*)out,
                                                  ldo);
      break;
    case RB_C64:
      jac_remap_kernel<cfloat><<<g, 256, 0, st>>>((const cfloat*)J, rows, ldj, map_ptr, map_idx, map_w, nq,
                                                   (cfloat*)out, ldo);
      break;
    case RB_F64:
      jac_remap_kernel<double><<<g, 256, 0, st>>>((const double*)J, rows, ldj, map_ptr, map_idx, map_w, nq,
                                                   (double*)out, ldo);
      break;
    case RB_C128:
      jac_remap_kernel<cdouble><<<g, 256, 0, st>>>((const cdouble*)J, rows, ldj, map_ptr, map_idx, map_w, nq,
                                                    (cdouble*)out, ldo);
      break;
    default:
      return fail(RB_EARG, "rb_jac_remap: bad kind");
  }
  RB_LAUNCH_CHECK();
  return RB_OK;
}

int rb_jac_block(const void* src, int32_t kind, int64_t rows, int64_t cols, int64_t lds, double scale_re,
                 double scale_im, const double* rowscale, float* dst, int64_t ldd, int64_t row_re, int64_t row_im,
                 int64_t col0, void* stream) {
  if (!src || !dst || rows < 0 || cols < 0 || lds < cols || col0 < 0 || col0 + cols > ldd || row_re < 0)
    return fail(RB_EARG, "rb_jac_block: bad arguments");
  if (rows * cols == 0) return RB_OK;
  const unsigned g = (unsigned)std::min<int64_t>(ceil_div(rows * cols, 256), 148 * 64);
  cudaStream_t st = as_stream(stream);
  switch (kind) {
    case RB_F32:
      jac_block_kernel<float><<<g, 256, 0, st>>>((const float*)src, rows, cols, lds, scale_re, scale_im, rowscale,
                                                  dst, ldd, row_re, row_im, col0);
      break;
    case RB_C64:
      jac_block_kernel<cfloat><<<g, 256, 0, st>>>((const cfloat*)src, rows, cols, lds, scale_re, scale_im, rowscale,
                                                   dst, ldd, row_re, row_im, col0);
      break;
    default:
      return fail(RB_EARG, "rb_jac_block: kind must be RB_F32 or RB_C64");
  }
  RB_LAUNCH_CHECK();
  return RB_OK;
}

}  // extern "C"
