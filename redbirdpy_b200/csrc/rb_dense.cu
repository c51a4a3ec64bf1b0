// Dense FP64 pieces of the Gauss-Newton step (reginvunder,
// redbirdpy/recon.py:429-509 and _normalize_diag, recon.py:784-789):
//   H += lambda I, di = 1/sqrt(|diag H| + 1e-16), H <- di H di     (prepare)
//   H = L L^T, blocked right-looking Cholesky (64-wide panels; the
//   inverse of each diagonal block kept in its strict upper triangle)  (cholesky)
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

// Factor the nb x nb diagonal block at (j0, j0) (lower, L11) and form its
// inverse X = L11^-1.  256 threads; thread (j = tid / 4, q = tid % 4) owns
// column j, rows q, q + 4, ..., so the 4 owners of a column are 4 lanes of
// one warp and exchange through shuffles.  Column c is scaled by its owners
// (the pivot comes from the lane holding the diagonal), published to shared
// memory (two buffers, so one barrier per column), and every thread updates
// its entries right of c.  X is formed column by column by forward
// substitution (the 4 owners of column j sum their own rows' terms, fixed
// order) and stored transposed in the block's strict upper triangle:
// H[j0 + j][j0 + i] = X[i][j], i > j (the diagonal of X is 1 / L[i][i]).
// The panel solve and rb_chol_solve then apply X as a product.
__global__ void __launch_bounds__(256) potrf_diag_kernel(double* __restrict__ H, int64_t ldh, int64_t j0, int nb,
                                                         int* __restrict__ err) {
  __shared__ double col[2][kNB];
  __shared__ double Ls[kNB][kNB + 1];
  const int tid = threadIdx.x;
  const int j = tid >> 2, q = tid & 3;
  const int lane = tid & 31;
  const unsigned quad = 0xFu << (lane & ~3);
  double a[kNB / 4];
#pragma unroll
  for (int u = 0; u < kNB / 4; ++u) {
    const int i = q + 4 * u;
    a[u] = (i < nb && j < nb && i >= j) ? H[(j0 + i) * ldh + j0 + j] : 0.0;
  }
  for (int c = 0; c < nb; ++c) {
    double* cc = col[c & 1];
    if (j == c) {  // the 4 owners of column c (one quad of one warp)
      double d = 0.0;
#pragma unroll
      for (int u = 0; u < kNB / 4; ++u)
        if (q + 4 * u == c) d = a[u];
      d = __shfl_sync(quad, d, (lane & ~3) | (c & 3));
      const bool ok = d > 0.0 && isfinite(d);
      const double piv = ok ? sqrt(d) : 1.0;
      if (!ok && q == 0) atomicExch(err, (int)(j0 + c) + 1);
#pragma unroll
      for (int u = 0; u < kNB / 4; ++u) {
        const int i = q + 4 * u;
        if (i >= c && i < nb) {
          a[u] = (i == c) ? piv : a[u] / piv;
          cc[i] = a[u];
        }
      }
    }
    __syncthreads();
    if (j > c && j < nb) {
      const double lj = cc[j];
#pragma unroll
      for (int u = 0; u < kNB / 4; ++u) {
        const int i = q + 4 * u;
        if (i >= j && i < nb) a[u] = fma(-cc[i], lj, a[u]);
      }
    }
  }
  // L11 back to H (lower) and to shared memory for the inverse
#pragma unroll
  for (int u = 0; u < kNB / 4; ++u) {
    const int i = q + 4 * u;
    Ls[i][j] = (i >= j && i < nb && j < nb) ? a[u] : 0.0;
    if (i >= j && i < nb && j < nb) H[(j0 + i) * ldh + j0 + j] = a[u];
  }
  __syncthreads();
  // X = L11^-1, column j by the quad of column j: X[j][j] = 1 / L[j][j],
  // X[i][j] = -(sum_{k=j}^{i-1} L[i][k] X[k][j]) / L[i][i]
  double x[kNB / 4];
#pragma unroll
  for (int u = 0; u < kNB / 4; ++u) x[u] = 0.0;
  for (int i = 0; i < nb; ++i) {
    double part = 0.0;
#pragma unroll
    for (int u = 0; u < kNB / 4; ++u) {
      const int k = q + 4 * u;
      if (k >= j && k < i) part = fma(Ls[i][k], x[u], part);
    }
    part += __shfl_xor_sync(0xffffffffu, part, 1);
    part += __shfl_xor_sync(0xffffffffu, part, 2);
    if (i >= j && j < nb) {
      const double xi = (i == j) ? 1.0 / Ls[i][i] : -part / Ls[i][i];
#pragma unroll
      for (int u = 0; u < kNB / 4; ++u)
        if (q + 4 * u == i) x[u] = xi;
    }
  }
#pragma unroll
  for (int u = 0; u < kNB / 4; ++u) {
    const int i = q + 4 * u;
    if (i > j && i < nb && j < nb) H[(j0 + j) * ldh + j0 + i] = x[u];
  }
}

// X^T of a factored diagonal block in shared memory: Xt[t][c] = X[c][t]
// (t <= c; H's strict upper triangle of the block, 1 / L[c][c] on the
// diagonal, zero below)
__device__ __forceinline__ void load_inv_t(const double* __restrict__ H, int64_t ldh, int64_t j0, int nb,
                                           double (*Xt)[kNB + 1]) {
  for (int e = threadIdx.x; e < kNB * kNB; e += blockDim.x) {
    const int t = e / kNB, c = e % kNB;
    double v = 0.0;
    if (t < nb && c < nb) {
      if (c > t) v = H[(j0 + t) * ldh + j0 + c];
      else if (c == t) v = 1.0 / H[(j0 + t) * ldh + j0 + t];
    }
    Xt[t][c] = v;
  }
}

// L21 = A21 L11^-T = A21 X^T for the rows below the panel: a CTA takes 64
// rows (4 x 4 outputs per thread), sums t = 0..c in order, and writes its
// rows back in place
constexpr int kTrsmSmem = 2 * kNB * (kNB + 1) * (int)sizeof(double);  // dynamic: above the 48 KB static limit
__global__ void __launch_bounds__(256) trsm_panel_kernel(double* __restrict__ H, int64_t ldh, int64_t M, int64_t j0,
                                                         int nb) {
  extern __shared__ double tsm[];
  double(*Xt)[kNB + 1] = reinterpret_cast<double(*)[kNB + 1]>(tsm);
  double(*As)[kNB + 1] = Xt + kNB;
  const int tid = threadIdx.x;
  const int64_t r0 = j0 + nb + blockIdx.x * (int64_t)kNB;
  load_inv_t(H, ldh, j0, nb, Xt);
  for (int e = tid; e < kNB * kNB; e += blockDim.x) {
    const int i = e / kNB, t = e % kNB;
    As[i][t] = (r0 + i < M && t < nb) ? H[(r0 + i) * ldh + j0 + t] : 0.0;
  }
  __syncthreads();
  const int tr = (tid >> 4) * 4, tc = (tid & 15) * 4;
  double acc[4][4];
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) acc[u][v] = 0.0;
  const int tmax = min(nb, tc + 4);
  for (int t = 0; t < tmax; ++t) {
    double xa[4], xb[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) xa[u] = As[tr + u][t];
#pragma unroll
    for (int v = 0; v < 4; ++v) xb[v] = Xt[t][tc + v];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[u][v] = fma(xa[u], xb[v], acc[u][v]);
  }
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int64_t r = r0 + tr + u;
      const int c = tc + v;
      if (r < M && c < nb) H[r * ldh + j0 + c] = acc[u][v];
    }
}

// trailing update A22 -= L21 L21^T on 64 x 64 tiles of the lower triangle.
// 128 threads, 8 x 4 outputs each; the panel is staged k-major in two
// 32-column halves so that a thread's 8 (and 4) operands are consecutive in
// shared memory (16-byte loads; rows padded to 66 doubles).
// The update reaches columns below c_end only; with c_end < M (the columns
// of the rest of an outer block) the grid is 2-D, x the row tile and y the
// column tile, and tiles above the diagonal return at once.
constexpr int kSyrkThreads = 128;
__global__ void __launch_bounds__(kSyrkThreads) syrk_update_kernel(double* __restrict__ H, int64_t ldh, int64_t M,
                                                                   int64_t j0, int nb, int64_t c_end) {
  __shared__ __align__(16) double As[32][kNB + 2];
  __shared__ __align__(16) double Bs[32][kNB + 2];
  const int64_t s0 = j0 + nb;  // first trailing row
  int64_t ti, tj;
  if (c_end < M) {
    ti = blockIdx.x;
    tj = blockIdx.y;
    if (tj > ti) return;
  } else {
    // blockIdx.x enumerates lower tiles (ti >= tj) in row-major order
    int64_t t = blockIdx.x;
    ti = 0;
    while (t > ti) {
      t -= ti + 1;
      ++ti;
    }
    tj = t;
  }
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
      if (i < M && j < c_end && j <= i) H[i * ldh + j] -= acc[u][v];
    }
}

// The triangular solves of rb_chol_solve apply the diagonal blocks' inverses
// X (kept by rb_cholesky in each block's strict upper triangle):
// mode 0: y = X v (solves L_kk y = v), mode 1: y = X^T v (solves L_kk^T y = v).
// y = X v (mode 0) or X^T v (mode 1) of diagonal block k0 into shared memory,
// by all 256 threads of the block (a quad per output, fixed order), v read
// from src[k0 ..]
__device__ __forceinline__ void tri_block_apply(const double* __restrict__ L, int64_t ldh, int64_t k0, int nb,
                                                const double* __restrict__ src, int mode, double* v, double* y) {
  const int tid = threadIdx.x;
  const int i = tid >> 2, q = tid & 3;
  if (tid < nb) v[tid] = src[k0 + tid];
  __syncthreads();
  double s = 0.0;
  if (i < nb) {
    if (mode == 0) {
      for (int t = q; t <= i; t += 4)
        s = fma(t == i ? 1.0 / L[(k0 + i) * ldh + k0 + i] : L[(k0 + t) * ldh + k0 + i], v[t], s);
    } else {
      for (int t = i + q; t < nb; t += 4)
        s = fma(t == i ? 1.0 / L[(k0 + i) * ldh + k0 + i] : L[(k0 + i) * ldh + k0 + t], v[t], s);
    }
  }
  s += __shfl_xor_sync(0xffffffffu, s, 1);
  s += __shfl_xor_sync(0xffffffffu, s, 2);
  if (i < nb && q == 0) y[i] = s;
  __syncthreads();
}

// One forward step of L y = b, fused: every block solves diagonal block k0
// (y = X v, v = x[k0 ..]) itself, block 0 stores y in w, and each block
// subtracts L[r][k0 ..] y from its 8 rows r below the block (a warp per row).
__global__ void __launch_bounds__(256) fwd_solve_kernel(const double* __restrict__ L, int64_t ldh, int64_t M,
                                                        int64_t k0, int nb, double* __restrict__ x,
                                                        double* __restrict__ w) {
  __shared__ double v[kNB], y[kNB];
  tri_block_apply(L, ldh, k0, nb, x, 0, v, y);
  if (blockIdx.x == 0 && threadIdx.x < nb) w[k0 + threadIdx.x] = y[threadIdx.x];
  const int lane = threadIdx.x & 31;
  const int64_t r = k0 + nb + blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5);
  if (r >= M) return;
  double s = 0.0;
  for (int c = lane; c < nb; c += 32) s += L[r * ldh + k0 + c] * y[c];
  s = warp_sum(s);
  if (lane == 0) x[r] -= s;
}

// One backward step of L^T x = y, fused: every block solves diagonal block
// k0 (v = w[k0 ..], the forward solution less the later blocks' terms),
// block 0 stores the result in x, and each block subtracts L[k0 + r][j] y[r]
// from its 32 columns j < k0 of w (8 warps over the block's rows, summed in
// a fixed order).
__global__ void __launch_bounds__(256) bwd_solve_kernel(const double* __restrict__ L, int64_t ldh, int64_t k0, int nb,
                                                        double* __restrict__ w, double* __restrict__ x) {
  __shared__ double v[kNB], y[kNB], part[8][32];
  tri_block_apply(L, ldh, k0, nb, w, 1, v, y);
  if (blockIdx.x == 0 && threadIdx.x < nb) x[k0 + threadIdx.x] = y[threadIdx.x];
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  const int64_t j = blockIdx.x * 32 + lane;
  double s = 0.0;
  if (j < k0)
    for (int r = wp; r < nb; r += 8) s = fma(L[(k0 + r) * ldh + j], y[r], s);
  part[wp][lane] = s;
  __syncthreads();
  if (wp == 0 && j < k0) {
    double t = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) t += part[q][lane];
    w[j] -= t;
  }
}

constexpr int kGemvSlabs = 16;

__device__ __forceinline__ double jval(float v) { return v; }
__device__ __forceinline__ double jval(__nv_bfloat16 v) { return __bfloat162float(v); }

// four consecutive entries of a row (16-byte FP32 / 8-byte BF16 loads)
__device__ __forceinline__ void ld4(const float* p, double (&v)[4]) {
  const float4 x = __ldcs(reinterpret_cast<const float4*>(p));
  v[0] = x.x;
  v[1] = x.y;
  v[2] = x.z;
  v[3] = x.w;
}
__device__ __forceinline__ void ld4(const __nv_bfloat16* p, double (&v)[4]) {
  const uint2 x = __ldcs(reinterpret_cast<const uint2*>(p));
  const __nv_bfloat162 a = *reinterpret_cast<const __nv_bfloat162*>(&x.x);
  const __nv_bfloat162 b = *reinterpret_cast<const __nv_bfloat162*>(&x.y);
  v[0] = __bfloat162float(a.x);
  v[1] = __bfloat162float(a.y);
  v[2] = __bfloat162float(b.x);
  v[3] = __bfloat162float(b.y);
}

// J stored as FP32 or BF16 (JT).  A thread owns 4 consecutive columns (one
// vector load per row; ldj % 4 == 0 keeps it aligned and inside the padded
// row) and sums its slab's rows in 4 interleaved partial sums per column
// (rows m = 0, 1, 2, 3 mod 4), added as (s0 + s1) + (s2 + s3).
template <typename JT>
__global__ void gemv_t_part_kernel(const JT* __restrict__ J, int64_t M, int64_t K, int64_t ldj,
                                   const double* __restrict__ y, double* __restrict__ part) {
  const int64_t k = 4 * (blockIdx.x * (int64_t)blockDim.x + threadIdx.x);
  if (k >= K) return;
  const int64_t rows = (M + gridDim.y - 1) / gridDim.y;
  const int64_t m0 = blockIdx.y * rows, m1 = min(M, m0 + rows);
  double s[4][4];
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int u = 0; u < 4; ++u) s[j][u] = 0.0;
  int64_t m = m0;
  for (; m + 3 < m1; m += 4) {
    double v[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u) ld4(J + (m + u) * ldj + k, v[u]);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const double ym = y[m + u];
#pragma unroll
      for (int j = 0; j < 4; ++j) s[j][u] = fma(v[u][j], ym, s[j][u]);
    }
  }
  for (; m < m1; ++m) {
    double v[4];
    ld4(J + m * ldj + k, v);
    const double ym = y[m];
#pragma unroll
    for (int j = 0; j < 4; ++j) s[j][0] = fma(v[j], ym, s[j][0]);
  }
#pragma unroll
  for (int j = 0; j < 4; ++j)
    if (k + j < K) part[blockIdx.y * K + k + j] = (s[j][0] + s[j][1]) + (s[j][2] + s[j][3]);
}

__global__ void gemv_t_sum_kernel(const double* __restrict__ part, int slabs, int64_t K, double alpha, double beta,
                                  double* __restrict__ out) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= K) return;
  double s = 0.0;
  for (int b = 0; b < slabs; ++b) s += part[b * K + k];
  out[k] = alpha * s + (beta != 0.0 ? beta * out[k] : 0.0);
}

// out[m] = alpha sum_k J[m][k] x[k] + beta out[m] for 4 rows per block: the
// FP32 (or BF16) rows stream from DRAM once, x (FP64) from L2 once per 4 rows;
// each thread keeps 4 partial sums per row (k chunks of 4), then a fixed-order
// block reduction: the result is the same bits on every run.
constexpr int kGemvNRows = 4;
template <typename JT>
__global__ void __launch_bounds__(256) gemv_n_kernel(const JT* __restrict__ J, int64_t M, int64_t K, int64_t ldj,
                                                     const double* __restrict__ x, double alpha, double beta,
                                                     double* __restrict__ out) {
  __shared__ double red[kGemvNRows][8];
  const int64_t m0 = (int64_t)blockIdx.x * kGemvNRows;
  double s[kGemvNRows];
#pragma unroll
  for (int r = 0; r < kGemvNRows; ++r) s[r] = 0.0;
  for (int64_t k = 4 * (int64_t)threadIdx.x; k < K; k += 4 * (int64_t)blockDim.x) {
    double xv[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) xv[j] = (k + j < K) ? x[k + j] : 0.0;
#pragma unroll
    for (int r = 0; r < kGemvNRows; ++r) {
      if (m0 + r < M) {
        double v[4];
        ld4(J + (m0 + r) * ldj + k, v);  // padded row: entries past K are read, then skipped
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (k + j < K) s[r] = fma(v[j], xv[j], s[r]);
      }
    }
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int r = 0; r < kGemvNRows; ++r) {
    const double t = warp_sum(s[r]);
    if (lane == 0) red[r][w] = t;
  }
  __syncthreads();
  if (threadIdx.x < kGemvNRows && m0 + threadIdx.x < M) {
    double t = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += red[threadIdx.x][q];
    const int64_t m = m0 + threadIdx.x;
    out[m] = alpha * t + (beta != 0.0 ? beta * out[m] : 0.0);
  }
}

// per-block partial sums of x . y (FP64), fixed order
__global__ void dot_part_kernel(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                                double* __restrict__ part) {
  __shared__ double red[32];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s = fma(x[i], y[i], s);
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
    t = warp_sum(t);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
  }
}

__global__ void axpby_kernel(int64_t n, double a, const double* __restrict__ x, double b, double* __restrict__ y) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) y[i] = a * x[i] + (b != 0.0 ? b * y[i] : 0.0);
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

// out[m] = sum_k J[m][k]^2 in FP64: a block per row, a fixed-order
// reduction (the diagonal of J J^T without the tensor cores' input rounding)
// With bf != NULL the pass also writes the rows rounded to BF16 (row stride
// ldb, the padding columns K..ldb-1 zeroed): the operand of a BF16 product
// whose refinement runs over the FP32 rows.
template <typename JT>
__global__ void row_sumsq_kernel(const JT* __restrict__ J, int64_t M, int64_t K, int64_t ldj,
                                 double* __restrict__ out, __nv_bfloat16* __restrict__ bf, int64_t ldb) {
  __shared__ double red[32];
  for (int64_t m = blockIdx.x; m < M; m += gridDim.x) {
    double s = 0.0;
    for (int64_t k = threadIdx.x; k < K; k += blockDim.x) {
      const JT x = J[m * ldj + k];
      const double v = jval(x);
      s += v * v;
      if (bf) bf[m * ldb + k] = __float2bfloat16_rn((float)v);
    }
    if (bf)
      for (int64_t k = K + threadIdx.x; k < ldb; k += blockDim.x) bf[m * ldb + k] = __float2bfloat16_rn(0.f);
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
      double t = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
      t = warp_sum(t);
      if (threadIdx.x == 0) out[m] = t;
    }
    __syncthreads();
  }
}

// H[i][i] = alpha d[i]
__global__ void set_diag_kernel(double* __restrict__ H, int64_t M, int64_t ldh, const double* __restrict__ d,
                                double alpha) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < M) H[i * ldh + i] = alpha * d[i];
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
  RB_CUDA_TRY(cudaFuncSetAttribute(trsm_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrsmSmem));
  // Right-looking in outer blocks of kOuter columns: inside a block each
  // 64-wide panel is factored (diagonal block, panel solve) and updates only
  // the rest of the block's columns; the rows and columns right of the block
  // then take one update of depth kOuter.  The trailing matrix is read and
  // written once per outer block instead of once per panel.
  constexpr int64_t kOuter = 4 * kNB;
  for (int64_t J0 = 0; J0 < M; J0 += kOuter) {
    const int64_t bend = std::min<int64_t>(J0 + kOuter, M);
    for (int64_t j0 = J0; j0 < bend; j0 += kNB) {
      const int nb = (int)std::min<int64_t>(kNB, M - j0);
      potrf_diag_kernel<<<1, 256, 0, st>>>(H, ldh, j0, nb, err);
      RB_LAUNCH_CHECK();
      const int64_t rest = M - j0 - nb;
      if (rest <= 0) break;
      trsm_panel_kernel<<<(unsigned)ceil_div(rest, kNB), 256, kTrsmSmem, st>>>(H, ldh, M, j0, nb);
      RB_LAUNCH_CHECK();
      if (j0 + nb < bend) {  // the block's later panels
        const int64_t T = ceil_div(rest, kNB), Tc = ceil_div(bend - (j0 + nb), kNB);
        syrk_update_kernel<<<dim3((unsigned)T, (unsigned)Tc), kSyrkThreads, 0, st>>>(H, ldh, M, j0, nb, bend);
        RB_LAUNCH_CHECK();
      }
    }
    const int64_t rest = M - bend;
    if (rest <= 0) break;
    const int64_t T = ceil_div(rest, kNB);
    syrk_update_kernel<<<(unsigned)(T * (T + 1) / 2), kSyrkThreads, 0, st>>>(H, ldh, M, J0, (int)(bend - J0), M);
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
  // one launch per diagonal block and direction: each block of a launch
  // solves the 64 x 64 diagonal step itself and then its share of the update
  double* w = nullptr;  // the forward solution, consumed by the backward steps
  RB_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&w), sizeof(double) * M, st));
  for (int64_t k0 = 0; k0 < M; k0 += kNB) {  // L y = b
    const int nb = (int)std::min<int64_t>(kNB, M - k0);
    const int64_t rest = M - k0 - nb;
    fwd_solve_kernel<<<(unsigned)std::max<int64_t>(1, ceil_div(rest, 8)), 256, 0, st>>>(L, ldh, M, k0, nb, x, w);
    RB_LAUNCH_CHECK();
  }
  for (int64_t k0 = ((M - 1) / kNB) * kNB; k0 >= 0; k0 -= kNB) {  // L^T x = y
    const int nb = (int)std::min<int64_t>(kNB, M - k0);
    bwd_solve_kernel<<<(unsigned)std::max<int64_t>(1, ceil_div(k0, 32)), 256, 0, st>>>(L, ldh, k0, nb, w, x);
    RB_LAUNCH_CHECK();
  }
  RB_CUDA_TRY(cudaFreeAsync(w, st));
  return RB_OK;
}

size_t rb_gemv_t_work_bytes(int64_t K) { return (size_t)kGemvSlabs * K * sizeof(double) + 256; }

}  // extern "C"

template <typename JT>
static int gemv_t_run(const JT* J, int64_t M, int64_t K, int64_t ldj, const double* y, double alpha, double beta,
                      double* out, void* work, size_t work_bytes, void* stream) {
  if (!J || !y || !out || !work || M < 1 || K < 1 || ldj < K) return fail(RB_EARG, "rb_gemv_t: bad arguments");
  if (work_bytes < rb_gemv_t_work_bytes(K)) return fail(RB_EARG, "rb_gemv_t: workspace too small");
  if ((reinterpret_cast<uintptr_t>(J) & (4 * sizeof(JT) - 1)) || (ldj % 4))
    return fail(RB_EARG, "rb_gemv_t: J rows must start on %d-byte boundaries (aligned J, ldj %% 4 == 0)",
                (int)(4 * sizeof(JT)));
  cudaStream_t st = as_stream(stream);
  const int slabs = (int)std::min<int64_t>(kGemvSlabs, M);
  double* part = reinterpret_cast<double*>(work);
  gemv_t_part_kernel<JT><<<dim3((unsigned)ceil_div(K, 4 * 256), (unsigned)slabs), 256, 0, st>>>(J, M, K, ldj, y,
                                                                                                part);
  RB_LAUNCH_CHECK();
  gemv_t_sum_kernel<<<(unsigned)ceil_div(K, 256), 256, 0, st>>>(part, slabs, K, alpha, beta, out);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

template <typename JT>
static int gemv_n_run(const JT* J, int64_t M, int64_t K, int64_t ldj, const double* x, double alpha, double beta,
                      double* out, void* stream) {
  if (!J || !x || !out || M < 1 || K < 1 || ldj < K) return fail(RB_EARG, "rb_gemv_n: bad arguments");
  if ((reinterpret_cast<uintptr_t>(J) & (4 * sizeof(JT) - 1)) || (ldj % 4) || ldj < ceil_div(K, 4) * 4)
    return fail(RB_EARG, "rb_gemv_n: J rows must start on %d-byte boundaries and hold K rounded up to 4 entries",
                (int)(4 * sizeof(JT)));
  gemv_n_kernel<JT><<<(unsigned)ceil_div(M, kGemvNRows), 256, 0, as_stream(stream)>>>(J, M, K, ldj, x, alpha, beta,
                                                                                       out);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

extern "C" {

int rb_gemv_n(const float* J, int64_t M, int64_t K, int64_t ldj, const double* x, double alpha, double beta,
              double* out, void* stream) {
  return gemv_n_run(J, M, K, ldj, x, alpha, beta, out, stream);
}

int rb_gemv_n_bf16(const void* J, int64_t M, int64_t K, int64_t ldj, const double* x, double alpha, double beta,
                   double* out, void* stream) {
  return gemv_n_run(reinterpret_cast<const __nv_bfloat16*>(J), M, K, ldj, x, alpha, beta, out, stream);
}

size_t rb_dot_work_bytes(void) { return 64 * sizeof(double) + 256; }

int rb_dot(int64_t n, const double* x, const double* y, double* out, void* work, size_t work_bytes, void* stream) {
  if (!x || !y || !out || !work || n < 1) return fail(RB_EARG, "rb_dot: bad arguments");
  if (work_bytes < rb_dot_work_bytes()) return fail(RB_EARG, "rb_dot: workspace too small");
  cudaStream_t st = as_stream(stream);
  const int blocks = (int)std::min<int64_t>(64, ceil_div(n, 256));
  double* part = reinterpret_cast<double*>(work);
  dot_part_kernel<<<blocks, 256, 0, st>>>(n, x, y, part);
  RB_LAUNCH_CHECK();
  sum_parts_kernel<<<1, 64, 0, st>>>(part, blocks, out);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

int rb_axpby(int64_t n, double a, const double* x, double b, double* y, void* stream) {
  if (!x || !y || n < 0) return fail(RB_EARG, "rb_axpby: bad arguments");
  if (n == 0) return RB_OK;
  axpby_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, as_stream(stream)>>>(n, a, x, b, y);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

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

template <typename JT>
static int row_sumsq_run(const JT* J, int64_t M, int64_t K, int64_t ldj, double* rows, double* total, void* stream,
                         __nv_bfloat16* bf = nullptr, int64_t ldb = 0) {
  if (!J || !rows || M < 1 || K < 1 || ldj < K || M > INT32_MAX) return fail(RB_EARG, "rb_row_sumsq: bad arguments");
  if (bf && (ldb < K || ldb % 8)) return fail(RB_EARG, "rb_row_sumsq_to_bf16: ldb must be >= K and a multiple of 8");
  cudaStream_t st = as_stream(stream);
  const unsigned nb = (unsigned)std::min<int64_t>(M, 148 * 16);
  row_sumsq_kernel<JT><<<nb, 256, 0, st>>>(J, M, K, ldj, rows, bf, ldb);
  RB_LAUNCH_CHECK();
  if (total) {
    sum_parts_kernel<<<1, 1024, 0, st>>>(rows, (int)M, total);
    RB_LAUNCH_CHECK();
  }
  return RB_OK;
}

extern "C" {

int rb_row_sumsq(const float* J, int64_t M, int64_t K, int64_t ldj, double* rows, double* total, void* stream) {
  return row_sumsq_run(J, M, K, ldj, rows, total, stream);
}

int rb_row_sumsq_bf16(const void* J, int64_t M, int64_t K, int64_t ldj, double* rows, double* total,
                      void* stream) {
  return row_sumsq_run(reinterpret_cast<const __nv_bfloat16*>(J), M, K, ldj, rows, total, stream);
}

int rb_row_sumsq_to_bf16(const float* J, int64_t M, int64_t K, int64_t ldj, double* rows, double* total, void* bf,
                         int64_t ldb, void* stream) {
  if (!bf) return fail(RB_EARG, "rb_row_sumsq_to_bf16: null output");
  return row_sumsq_run(J, M, K, ldj, rows, total, stream, reinterpret_cast<__nv_bfloat16*>(bf), ldb);
}

int rb_set_diag(double* H, int64_t M, int64_t ldh, const double* d, double alpha, void* stream) {
  if (!H || !d || M < 1 || ldh < M) return fail(RB_EARG, "rb_set_diag: bad arguments");
  set_diag_kernel<<<(unsigned)ceil_div(M, 256), 256, 0, as_stream(stream)>>>(H, M, ldh, d, alpha);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

}  // extern "C"
