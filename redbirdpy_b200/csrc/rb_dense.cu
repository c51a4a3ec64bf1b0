// Dense FP64 pieces of the Gauss-Newton step (reginvunder,
// redbirdpy/recon.py:429-509 and _normalize_diag, recon.py:784-789):
//   H += lambda I, di = 1/sqrt(|diag H| + 1e-16), H <- di H di     (prepare)
//   H = L L^T, blocked right-looking Cholesky (64-wide panels)      (cholesky)
//   L L^T x = b                                                    (chol_solve)
//   out = alpha * J^T y   (J FP32 M x K rows, y FP64)              (gemv_t)
//   sum(J^2)              (Frobenius block scaling, recon.py:235)   (sumsq)
#include <algorithm>

#include <cuda_bf16.h>

#include "rb_common.cuh"

namespace rb {

constexpr int kNB = 64;  // panel width

__global__ void prep_diag_kernel(double* __restrict__ H, int64_t M, int64_t ldh, double lam, double* __restrict__ di) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= M) return;
  const double d = H[i * ldh + i] + lam;
  H[i * ldh + i] = d;
  di[i] = 1.0 / sqrt(fabs(d) + 1e-16);
}

__global__ void prep_scale_kernel(double* __restrict__ H, int64_t M, int64_t ldh, const double* __restrict__ di) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t i = blockIdx.y;
  if (j >= M) return;
  H[i * ldh + j] *= di[i] * di[j];
}

// Stage the lower triangle of the nb x nb block at (r0, c0) of H into
// shared memory (zeros above the diagonal), all loads issued before the
// stores so that they overlap (the block is read once from L2/HBM).
template <int LD>
__device__ __forceinline__ void load_lower(const double* __restrict__ H, int64_t ldh, int64_t r0, int64_t c0, int nb,
                                           double (*A)[LD]) {
  constexpr int kPer = 16;
  for (int e0 = threadIdx.x; e0 < kNB * kNB; e0 += kPer * blockDim.x) {
    double v[kPer];
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const int e = e0 + u * blockDim.x, i = e / kNB, j = e % kNB;
      v[u] = (e < kNB * kNB && i < nb && j <= i) ? H[(r0 + i) * ldh + c0 + j] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const int e = e0 + u * blockDim.x;
      if (e < kNB * kNB) A[e / kNB][e % kNB] = v[u];
    }
  }
}

// factor the nb x nb diagonal block at (j0, j0) in shared memory (lower)
__global__ void potrf_diag_kernel(double* __restrict__ H, int64_t ldh, int64_t j0, int nb, int* __restrict__ err) {
  __shared__ double A[kNB][kNB + 1];
  const int tid = threadIdx.x, nt = blockDim.x;
  load_lower<kNB + 1>(H, ldh, j0, j0, nb, A);
  __syncthreads();
  for (int c = 0; c < nb; ++c) {
    __shared__ double piv;
    if (tid == 0) {
      const double d = A[c][c];
      if (!(d > 0.0) || !isfinite(d)) {
        atomicExch(err, (int)(j0 + c) + 1);
        piv = 1.0;
      } else {
        piv = sqrt(d);
      }
      A[c][c] = piv;
    }
    __syncthreads();
    for (int i = c + 1 + tid; i < nb; i += nt) A[i][c] /= piv;
    __syncthreads();
    // trailing update of the lower part: A[i][j] -= A[i][c] A[j][c], c < j <= i
    const int m = nb - c - 1;
    for (int e = tid; e < m * m; e += nt) {
      const int i = c + 1 + e / m, j = c + 1 + e % m;
      if (j <= i) A[i][j] -= A[i][c] * A[j][c];
    }
    __syncthreads();
  }
  for (int e = tid; e < nb * nb; e += nt) {
    const int i = e / nb, j = e % nb;
    if (j <= i) H[(j0 + i) * ldh + j0 + j] = A[i][j];
  }
}

// L21 = A21 L11^{-T}: one thread per row below the panel, row in smem
__global__ void trsm_panel_kernel(double* __restrict__ H, int64_t ldh, int64_t M, int64_t j0, int nb) {
  __shared__ double L[kNB][kNB + 1];
  extern __shared__ double xs[];  // [kNB][blockDim.x]
  const int tid = threadIdx.x, nt = blockDim.x;
  load_lower<kNB + 1>(H, ldh, j0, j0, nb, L);
  __syncthreads();
  const int64_t r = j0 + nb + blockIdx.x * (int64_t)nt + tid;
  if (r >= M) return;
  double* row = H + r * ldh + j0;
  // the row itself, loaded up front
  for (int c = 0; c < nb; ++c) xs[c * nt + tid] = row[c];
  for (int c = 0; c < nb; ++c) {
    double s = xs[c * nt + tid];
    for (int t = 0; t < c; ++t) s -= xs[t * nt + tid] * L[c][t];
    xs[c * nt + tid] = s / L[c][c];
  }
  for (int c = 0; c < nb; ++c) row[c] = xs[c * nt + tid];
}

// trailing update A22 -= L21 L21^T on 64 x 64 tiles of the lower triangle.
// 128 threads, 8 x 4 outputs each; the panel is staged k-major in two
// 32-column halves so that a thread's 8 (and 4) operands are consecutive in
// shared memory (16-byte loads; rows padded to 66 doubles).
constexpr int kSyrkThreads = 128;
__global__ void __launch_bounds__(kSyrkThreads) syrk_update_kernel(double* __restrict__ H, int64_t ldh, int64_t M,
                                                                   int64_t j0, int nb) {
  __shared__ __align__(16) double As[32][kNB + 2];
  __shared__ __align__(16) double Bs[32][kNB + 2];
  const int64_t s0 = j0 + nb;  // first trailing row
  // blockIdx.x enumerates lower tiles (ti >= tj) in row-major order
  int64_t t = blockIdx.x, ti = 0;
  while (t > ti) {
    t -= ti + 1;
    ++ti;
  }
  const int64_t tj = t;
  const int64_t r0 = s0 + ti * kNB, c0 = s0 + tj * kNB;
  const int tid = threadIdx.x;
  const int tr = (tid >> 4) * 8, tc = (tid & 15) * 4;
  double acc[8][4];
#pragma unroll
  for (int u = 0; u < 8; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) acc[u][v] = 0.0;
  for (int k0 = 0; k0 < nb; k0 += 32) {
    const int kc = min(32, nb - k0);
    __syncthreads();
#pragma unroll 4
    for (int e = tid; e < kNB * 32; e += kSyrkThreads) {
      const int i = e >> 5, k = e & 31;
      As[k][i] = (r0 + i < M && k < kc) ? H[(r0 + i) * ldh + j0 + k0 + k] : 0.0;
      Bs[k][i] = (c0 + i < M && k < kc) ? H[(c0 + i) * ldh + j0 + k0 + k] : 0.0;
    }
    __syncthreads();
    for (int k = 0; k < kc; ++k) {
      double a[8], b[4];
      const double2* pa = reinterpret_cast<const double2*>(&As[k][tr]);
      const double2* pb = reinterpret_cast<const double2*>(&Bs[k][tc]);
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const double2 x = pa[u];
        a[2 * u] = x.x;
        a[2 * u + 1] = x.y;
      }
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const double2 x = pb[u];
        b[2 * u] = x.x;
        b[2 * u + 1] = x.y;
      }
#pragma unroll
      for (int u = 0; u < 8; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = fma(a[u], b[v], acc[u][v]);
    }
  }
#pragma unroll
  for (int u = 0; u < 8; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int64_t i = r0 + tr + u, j = c0 + tc + v;
      if (i < M && j < M && j <= i) H[i * ldh + j] -= acc[u][v];
    }
}

// forward / backward substitution on one 64-block (single CTA)
// mode 0: solve L_kk y = x (lower), mode 1: solve L_kk^T y = x
__global__ void tri_block_kernel(const double* __restrict__ L, int64_t ldh, int64_t k0, int nb, double* __restrict__ x,
                                 int mode) {
  __shared__ double Lb[kNB][kNB + 1];
  __shared__ double v[kNB];
  const int tid = threadIdx.x;
  load_lower<kNB + 1>(L, ldh, k0, k0, nb, Lb);
  if (tid < nb) v[tid] = x[k0 + tid];
  __syncthreads();
  if (tid < 32) {  // one warp: each step's dot product across the lanes
    const int lane = tid;
    if (mode == 0) {
      for (int c = 0; c < nb; ++c) {
        double s = 0.0;
        for (int t = lane; t < c; t += 32) s += Lb[c][t] * v[t];
        s = warp_sum(s);
        if (lane == 0) v[c] = (v[c] - s) / Lb[c][c];
        __syncwarp();
      }
    } else {
      for (int c = nb - 1; c >= 0; --c) {
        double s = 0.0;
        for (int t = c + 1 + lane; t < nb; t += 32) s += Lb[t][c] * v[t];
        s = warp_sum(s);
        if (lane == 0) v[c] = (v[c] - s) / Lb[c][c];
        __syncwarp();
      }
    }
  }
  __syncthreads();
  if (tid < nb) x[k0 + tid] = v[tid];
}

// forward: x[r] -= sum_{c in block} L[r][k0+c] x[k0+c] for r >= k0+nb (warp per row)
__global__ void fwd_update_kernel(const double* __restrict__ L, int64_t ldh, int64_t M, int64_t k0, int nb,
                                  double* __restrict__ x) {
  const int lane = threadIdx.x & 31;
  const int64_t r = k0 + nb + blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5);
  if (r >= M) return;
  double s = 0.0;
  for (int c = lane; c < nb; c += 32) s += L[r * ldh + k0 + c] * x[k0 + c];
  s = warp_sum(s);
  if (lane == 0) x[r] -= s;
}

// backward: x[j] -= sum_{r in block} L[k0+r][j] x[k0+r] for j < k0 (thread per column)
__global__ void bwd_update_kernel(const double* __restrict__ L, int64_t ldh, int64_t k0, int nb, double* __restrict__ x) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= k0) return;
  double s = 0.0;
  for (int r = 0; r < nb; ++r) s += L[(k0 + r) * ldh + j] * x[k0 + r];
  x[j] -= s;
}

// out[k] = alpha * sum_m J[m][k] y[m] + beta out[k]   (coalesced along k).
// Rows are split over gridDim.y slabs; each slab writes a partial sum and the
// last kernel adds the slabs in fixed order (deterministic, no atomics).
constexpr int kGemvSlabs = 16;

__device__ __forceinline__ double jval(float v) { return v; }
__device__ __forceinline__ double jval(__nv_bfloat16 v) { return __bfloat162float(v); }

// J stored as FP32 or BF16 (JT)
template <typename JT>
__global__ void gemv_t_part_kernel(const JT* __restrict__ J, int64_t M, int64_t K, int64_t ldj,
                                   const double* __restrict__ y, double* __restrict__ part) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= K) return;
  const int64_t rows = (M + gridDim.y - 1) / gridDim.y;
  const int64_t m0 = blockIdx.y * rows, m1 = min(M, m0 + rows);
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  int64_t m = m0;
  for (; m + 3 < m1; m += 4) {
    s0 = fma(jval(J[m * ldj + k]), y[m], s0);
    s1 = fma(jval(J[(m + 1) * ldj + k]), y[m + 1], s1);
    s2 = fma(jval(J[(m + 2) * ldj + k]), y[m + 2], s2);
    s3 = fma(jval(J[(m + 3) * ldj + k]), y[m + 3], s3);
  }
  for (; m < m1; ++m) s0 = fma(jval(J[m * ldj + k]), y[m], s0);
  part[blockIdx.y * K + k] = (s0 + s1) + (s2 + s3);
}

__global__ void gemv_t_sum_kernel(const double* __restrict__ part, int slabs, int64_t K, double alpha, double beta,
                                  double* __restrict__ out) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= K) return;
  double s = 0.0;
  for (int b = 0; b < slabs; ++b) s += part[b * K + k];
  out[k] = alpha * s + (beta != 0.0 ? beta * out[k] : 0.0);
}

// per-block partial sums of J^2
template <typename JT>
__global__ void sumsq_kernel(const JT* __restrict__ J, int64_t M, int64_t K, int64_t ldj,
                             double* __restrict__ part) {
  __shared__ double red[32];
  double s = 0.0;
  for (int64_t m = blockIdx.x; m < M; m += gridDim.x)
    for (int64_t k = threadIdx.x; k < K; k += blockDim.x) {
      const double v = jval(J[m * ldj + k]);
      s += v * v;
    }
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
    t = warp_sum(t);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
  }
}

__global__ void sum_parts_kernel(const double* __restrict__ part, int n, double* __restrict__ out) {
  __shared__ double red[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += part[i];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
    t = warp_sum(t);
    if (threadIdx.x == 0) *out = t;
  }
}

__global__ void vec_mul_kernel(const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out,
                               int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = a[i] * b[i];
}

// hi = tf32(J) rounded to nearest (in place), lo = J - hi
__global__ void split_tf32_kernel(float* __restrict__ J, float* __restrict__ lo, int64_t M, int64_t K, int64_t ldj) {
  for (int64_t m = blockIdx.y; m < M; m += gridDim.y)
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < K; k += (int64_t)gridDim.x * blockDim.x) {
      const float v = J[m * ldj + k];
      uint32_t h;
      asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(v));
      const float hv = __uint_as_float(h);
      J[m * ldj + k] = hv;
      lo[m * ldj + k] = v - hv;
    }
}

}  // namespace rb

using namespace rb;

extern "C" {

int rb_reginv_prepare(double* H, int64_t M, int64_t ldh, double lambda, double* di, void* stream) {
  if (!H || !di || M < 1 || ldh < M) return fail(RB_EARG, "rb_reginv_prepare: bad arguments");
  if (M > 65535) return fail(RB_ESIZE, "rb_reginv_prepare: at most 65535 rows");
  cudaStream_t st = as_stream(stream);
  prep_diag_kernel<<<(unsigned)ceil_div(M, 256), 256, 0, st>>>(H, M, ldh, lambda, di);
  RB_LAUNCH_CHECK();
  prep_scale_kernel<<<dim3((unsigned)ceil_div(M, 256), (unsigned)M), 256, 0, st>>>(H, M, ldh, di);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

size_t rb_cholesky_work_bytes(void) { return 256; }

int rb_cholesky(double* H, int64_t M, int64_t ldh, void* work, size_t work_bytes, void* stream) {
  if (!H || !work || M < 1 || ldh < M) return fail(RB_EARG, "rb_cholesky: bad arguments");
  if (work_bytes < rb_cholesky_work_bytes()) return fail(RB_EARG, "rb_cholesky: workspace too small");
  if (M > 65535 * 32) return fail(RB_ESIZE, "rb_cholesky: matrix too large");
  cudaStream_t st = as_stream(stream);
  int* err = reinterpret_cast<int*>(work);
  RB_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), st));
  const int tthreads = 64;
  const int trsm_smem = (int)(kNB * tthreads * sizeof(double));  // + 33 KB static: opt in above 48 KB
  RB_CUDA_TRY(cudaFuncSetAttribute(trsm_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, trsm_smem));
  for (int64_t j0 = 0; j0 < M; j0 += kNB) {
    const int nb = (int)std::min<int64_t>(kNB, M - j0);
    potrf_diag_kernel<<<1, 256, 0, st>>>(H, ldh, j0, nb, err);
    RB_LAUNCH_CHECK();
    const int64_t rest = M - j0 - nb;
    if (rest <= 0) break;
    trsm_panel_kernel<<<(unsigned)ceil_div(rest, tthreads), tthreads, trsm_smem, st>>>(
        H, ldh, M, j0, nb);
    RB_LAUNCH_CHECK();
    const int64_t T = ceil_div(rest, kNB);
    syrk_update_kernel<<<(unsigned)(T * (T + 1) / 2), kSyrkThreads, 0, st>>>(H, ldh, M, j0, nb);
    RB_LAUNCH_CHECK();
  }
  int herr = 0;
  RB_CUDA_TRY(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  RB_CUDA_TRY(cudaStreamSynchronize(st));
  if (herr) return fail(RB_ENOTSPD, "rb_cholesky: non-positive pivot at row %d", herr - 1);
  return RB_OK;
}

int rb_chol_solve(const double* L, int64_t M, int64_t ldh, double* x, void* stream) {
  if (!L || !x || M < 1 || ldh < M) return fail(RB_EARG, "rb_chol_solve: bad arguments");
  cudaStream_t st = as_stream(stream);
  for (int64_t k0 = 0; k0 < M; k0 += kNB) {  // L y = b
    const int nb = (int)std::min<int64_t>(kNB, M - k0);
    tri_block_kernel<<<1, 256, 0, st>>>(L, ldh, k0, nb, x, 0);
    const int64_t rest = M - k0 - nb;
    if (rest > 0) fwd_update_kernel<<<(unsigned)ceil_div(rest, 8), 256, 0, st>>>(L, ldh, M, k0, nb, x);
    RB_LAUNCH_CHECK();
  }
  for (int64_t k0 = ((M - 1) / kNB) * kNB; k0 >= 0; k0 -= kNB) {  // L^T x = y
    const int nb = (int)std::min<int64_t>(kNB, M - k0);
    tri_block_kernel<<<1, 256, 0, st>>>(L, ldh, k0, nb, x, 1);
    if (k0 > 0) bwd_update_kernel<<<(unsigned)ceil_div(k0, 256), 256, 0, st>>>(L, ldh, k0, nb, x);
    RB_LAUNCH_CHECK();
  }
  return RB_OK;
}

size_t rb_gemv_t_work_bytes(int64_t K) { return (size_t)kGemvSlabs * K * sizeof(double) + 256; }

}  // extern "C"

template <typename JT>
static int gemv_t_run(const JT* J, int64_t M, int64_t K, int64_t ldj, const double* y, double alpha, double beta,
                      double* out, void* work, size_t work_bytes, void* stream) {
  if (!J || !y || !out || !work || M < 1 || K < 1 || ldj < K) return fail(RB_EARG, "rb_gemv_t: bad arguments");
  if (work_bytes < rb_gemv_t_work_bytes(K)) return fail(RB_EARG, "rb_gemv_t: workspace too small");
  cudaStream_t st = as_stream(stream);
  const int slabs = (int)std::min<int64_t>(kGemvSlabs, M);
  double* part = reinterpret_cast<double*>(work);
  gemv_t_part_kernel<JT><<<dim3((unsigned)ceil_div(K, 256), (unsigned)slabs), 256, 0, st>>>(J, M, K, ldj, y, part);
  RB_LAUNCH_CHECK();
  gemv_t_sum_kernel<<<(unsigned)ceil_div(K, 256), 256, 0, st>>>(part, slabs, K, alpha, beta, out);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

extern "C" {


int rb_gemv_t(const float* J, int64_t M, int64_t K, int64_t ldj, const double* y, double alpha, double beta,
              double* out, void* work, size_t work_bytes, void* stream) {
  return gemv_t_run(J, M, K, ldj, y, alpha, beta, out, work, work_bytes, stream);
}

int rb_gemv_t_bf16(const void* J, int64_t M, int64_t K, int64_t ldj, const double* y, double alpha, double beta,
                   double* out, void* work, size_t work_bytes, void* stream) {
  return gemv_t_run(reinterpret_cast<const __nv_bfloat16*>(J), M, K, ldj, y, alpha, beta, out, work, work_bytes,
                    stream);
}

int rb_vec_mul(const double* a, const double* b, double* out, int64_t n, void* stream) {
  if (!a || !b || !out || n < 0) return fail(RB_EARG, "rb_vec_mul: bad arguments");
  if (n == 0) return RB_OK;
  vec_mul_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, as_stream(stream)>>>(a, b, out, n);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

int rb_split_tf32(float* J, float* lo, int64_t M, int64_t K, int64_t ldj, void* stream) {
  if (!J || !lo || M < 1 || K < 1 || ldj < K) return fail(RB_EARG, "rb_split_tf32: bad arguments");
  dim3 g((unsigned)std::min<int64_t>(ceil_div(K, 256), 64), (unsigned)std::min<int64_t>(M, 4096));
  split_tf32_kernel<<<g, 256, 0, as_stream(stream)>>>(J, lo, M, K, ldj);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

size_t rb_sumsq_work_bytes(void) { return 148 * 8 * sizeof(double) + 256; }

}  // extern "C"

template <typename JT>
static int sumsq_run(const JT* J, int64_t M, int64_t K, int64_t ldj, double* out, void* work, size_t work_bytes,
                     void* stream) {
  if (!J || !out || !work || M < 1 || K < 1 || ldj < K) return fail(RB_EARG, "rb_sumsq: bad arguments");
  if (work_bytes < rb_sumsq_work_bytes()) return fail(RB_EARG, "rb_sumsq: workspace too small");
  cudaStream_t st = as_stream(stream);
  const int nb = 148 * 8;
  double* part = reinterpret_cast<double*>(work);
  sumsq_kernel<JT><<<nb, 256, 0, st>>>(J, M, K, ldj, part);
  RB_LAUNCH_CHECK();
  sum_parts_kernel<<<1, 1024, 0, st>>>(part, nb, out);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

extern "C" {


int rb_sumsq(const float* J, int64_t M, int64_t K, int64_t ldj, double* out, void* work, size_t work_bytes,
             void* stream) {
  return sumsq_run(J, M, K, ldj, out, work, work_bytes, stream);
}

int rb_sumsq_bf16(const void* J, int64_t M, int64_t K, int64_t ldj, double* out, void* work, size_t work_bytes,
                  void* stream) {
  return sumsq_run(reinterpret_cast<const __nv_bfloat16*>(J), M, K, ldj, out, work, work_bytes, stream);
}

}  // extern "C"
