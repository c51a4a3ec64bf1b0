// Dense FP64 pieces of the Gauss-Newton step (reginvunder,
// redbirdpy/recon.py:429-509 and _normalize_diag, recon.py:784-789):
//   H += lambda I, di = 1/sqrt(|diag H| + 1e-16), H <- di H di     (prepare)
//   H = L L^T, blocked right-looking Cholesky (64-wide panels; the
//   inverse of each diagonal block kept in its strict upper triangle)  (cholesky)
//   L L^T x = b                                                    (chol_solve)
//   out = alpha * J^T y   (J FP32 M x K rows, y FP64)              (gemv_t)
//   sum(J^2)              (Frobenius block scaling, recon.py:235)   (sumsq)
#include <algorithm>
#include <mutex>

#include <cuda_bf16.h>

#include "rb_common.cuh"
#include "rb_tc.cuh"

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

// Factor the nb x nb diagonal block at (j0, j0) (lower, L11) and form its
// inverse X = L11^-1.  256 threads; the block's lower triangle sits in
// shared memory.  Column c: every thread reads the pivot and forms its
// reciprocal square root itself (no hand-off), 64 threads scale the column,
// and after a barrier the rank-1 update of the columns right of c is spread
// over all threads (each owns the same ~9 entries of the triangle in every
// step).  X is then formed column by column by forward substitution (thread
// (j = tid / 4, q = tid % 4) owns column j, rows q, q + 4, ...; the quad's
// terms in four interleaved chains, added in fixed order) and stored
// transposed in the block's strict upper triangle:
// H[j0 + j][j0 + i] = X[i][j], i > j (the diagonal of X is 1 / L[i][i]).
// The panel solve and rb_chol_solve then apply X as a product.
constexpr int kTri = kNB * (kNB + 1) / 2;     // entries of the lower triangle
constexpr int kTriOwn = (kTri + 255) / 256;  // per thread
__global__ void __launch_bounds__(256) potrf_diag_kernel(double* __restrict__ H, int64_t ldh, int64_t j0, int nb,
                                                         int* __restrict__ err) {
  __shared__ double Ls[kNB][kNB + 1];
  __shared__ double rdiag[kNB];
  const int tid = threadIdx.x;
  for (int e = tid; e < kNB * kNB; e += 256) {
    const int i = e / kNB, j = e % kNB;
    Ls[i][j] = (i < nb && j <= i) ? H[(j0 + i) * ldh + j0 + j] : 0.0;
  }
  // owned entries e = tid + 256 v of the row-major lower triangle, (i, j)
  // packed as i * 256 + j (-1: none)
  int own[kTriOwn];
#pragma unroll
  for (int v = 0; v < kTriOwn; ++v) {
    const int e = tid + 256 * v;
    if (e < kTri) {
      int i = (int)((sqrtf(8.f * (float)e + 1.f) - 1.f) * 0.5f);
      while (i * (i + 1) / 2 > e) --i;
      while ((i + 1) * (i + 2) / 2 <= e) ++i;
      own[v] = i * 256 + (e - i * (i + 1) / 2);
    } else {
      own[v] = -1;
    }
  }
  __syncthreads();
  // Two columns per step (one barrier pair instead of two): with c and c + 1,
  // every thread forms both pivots itself; thread i scales its entry of
  // column c, takes column c's update of its entry of column c + 1 and
  // scales that; then the owned entries right of c + 1 take both updates,
  // column c's first.  Every entry sees the same operations in the same
  // order as in one column per step, so the factor is the same bits.
  // One reciprocal square root per column: the pivot is d / sqrt(d), and
  // the column is scaled by 1 / sqrt(d) (as LAPACK's dpotf2 scales by the
  // reciprocal).
  for (int c = 0; c < nb; c += 2) {
    if (c + 1 < nb) {
      const double d0 = Ls[c][c], a10 = Ls[c + 1][c], a11 = Ls[c + 1][c + 1];
      const bool ok0 = d0 > 0.0 && isfinite(d0);
      const double rp0 = ok0 ? rsqrt(d0) : 1.0;
      const double l10 = a10 * rp0;
      const double d1 = fma(-l10, l10, a11);
      const bool ok1 = d1 > 0.0 && isfinite(d1);
      const double rp1 = ok1 ? rsqrt(d1) : 1.0;
      if (tid == 0 && (!ok0 || !ok1)) atomicExch(err, (int)(j0 + c + (ok0 ? 1 : 0)) + 1);
      if (tid > c + 1 && tid < nb) {
        const double li0 = Ls[tid][c] * rp0;
        Ls[tid][c] = li0;
        Ls[tid][c + 1] = fma(-li0, l10, Ls[tid][c + 1]) * rp1;
      }
      __syncthreads();
      // every thread has read the pivots: their entries take L now (the
      // update below reads only the entries below them in columns c, c + 1)
      if (tid == c) Ls[c][c] = ok0 ? d0 * rp0 : 1.0;
      if (tid == c + 1) {
        Ls[c + 1][c] = l10;
        Ls[c + 1][c + 1] = ok1 ? d1 * rp1 : 1.0;
      }
#pragma unroll
      for (int v = 0; v < kTriOwn; ++v) {
        const int i = own[v] >> 8, j = own[v] & 255;
        if (own[v] >= 0 && j > c + 1 && i < nb)
          Ls[i][j] = fma(-Ls[i][c + 1], Ls[j][c + 1], fma(-Ls[i][c], Ls[j][c], Ls[i][j]));
      }
      __syncthreads();
    } else {  // the last column of an odd block
      const double d = Ls[c][c];
      const bool ok = d > 0.0 && isfinite(d);
      const double rp = ok ? rsqrt(d) : 1.0;
      if (tid == 0 && !ok) atomicExch(err, (int)(j0 + c) + 1);
      __syncthreads();
      if (tid == c) Ls[c][c] = ok ? d * rp : 1.0;
      __syncthreads();
    }
  }
  // L11 back to H (lower, whole rows)
  for (int e = tid; e < kNB * kNB; e += 256) {
    const int i = e / kNB, j = e % kNB;
    if (i < nb && j <= i) H[(j0 + i) * ldh + j0 + j] = Ls[i][j];
  }
  if (tid < nb) rdiag[tid] = 1.0 / Ls[tid][tid];  // the 64 reciprocals at once, off the chain below
  __syncthreads();
  // X = L11^-1, column j by the quad of column j: X[j][j] = 1 / L[j][j],
  // X[i][j] = -(sum_{k=j}^{i-1} L[i][k] X[k][j]) / L[i][i]
  const int j = tid >> 2, q = tid & 3;
  double x[kNB / 4];
#pragma unroll
  for (int u = 0; u < kNB / 4; ++u) x[u] = 0.0;
  for (int i = 0; i < nb; ++i) {
    double p[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int u = 0; u < kNB / 4; ++u) {
      const int k = q + 4 * u;
      if (k >= j && k < i) p[u & 3] = fma(Ls[i][k], x[u], p[u & 3]);
    }
    double part = (p[0] + p[1]) + (p[2] + p[3]);
    part += __shfl_xor_sync(0xffffffffu, part, 1);
    part += __shfl_xor_sync(0xffffffffu, part, 2);
    if (i >= j && j < nb) {
      const double ri = rdiag[i];
      const double xi = (i == j) ? ri : -part * ri;
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

// trailing update A22 -= L21 L21^T on 64 x 64 tiles of the lower triangle,
// on the FP64 tensor cores (mma.sync m8n8k4 .f64: D = A B + C, every
// product and sum in FP64).  128 threads: warp w owns the 32 x 32 quarter
// (w / 2, w % 2) of the tile as 4 x 4 MMA tiles of 8 x 8.  The panel's rows
// stream through shared memory in 32-column stages, double-buffered with
// cp.async (16-byte copies when every row start is 16-byte aligned, else
// 8-byte copies), rows kept k-contiguous with a stride of 36 doubles so that
// the fragment loads (8 rows x 4 k per warp) take the minimum two
// wavefronts.  Rows past M are zero-filled by the copy (source size 0).
// The panel is columns j0 .. j0 + nb; the tiles start at row and column s0
// and reach columns below c_end only.  With tri = 0 (a band of columns) the
// grid is 2-D, x the row tile and y the column tile, and tiles above the
// diagonal return at once; with tri = 1 (a whole trailing triangle)
// blockIdx.x enumerates the lower tiles.
constexpr int kSyrkThreads = 128;
constexpr int kSyK = 32;             // panel columns per stage
constexpr int kSyLd = kSyK + 4;      // shared row stride (doubles)
constexpr int kSyrkSmem = 2 * 2 * kNB * kSyLd * (int)sizeof(double);  // 2 stages x (A, B): 73,728 bytes

__device__ __forceinline__ void cp_async_f64(uint32_t dst, const double* src, int bytes, int src_bytes) {
  if (bytes == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void dmma_8x8x4(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// one stage of the panel: rows r0.. (A) and c0.. (B), columns kk.. of the
// panel (kc of them), into the shared buffers
template <int CH>
__device__ __forceinline__ void syrk_stage(const double* __restrict__ H, int64_t ldh, int64_t M, int64_t r0,
                                           int64_t c0, int64_t kcol, int kc, double* As, double* Bs) {
  constexpr int PER = kSyK * (int)sizeof(double) / CH;  // copies per row
  for (int e = threadIdx.x; e < 2 * kNB * PER; e += kSyrkThreads) {
    const int m = e / (kNB * PER), rem = e % (kNB * PER);
    const int i = rem / PER, kq = (rem % PER) * (CH / (int)sizeof(double));
    const int64_t row = (m == 0 ? r0 : c0) + i;
    const bool in = row < M && kq < kc;
    const double* src = in ? H + row * ldh + kcol + kq : H;
    double* dst = (m == 0 ? As : Bs) + i * kSyLd + kq;
    cp_async_f64(smem_u32(dst), src, CH, in ? min(CH, (kc - kq) * (int)sizeof(double)) : 0);
  }
}

template <int CH>
__global__ void __launch_bounds__(kSyrkThreads) syrk_update_kernel(double* __restrict__ H, int64_t ldh, int64_t M,
                                                                   int64_t j0, int nb, int64_t s0, int64_t c_end,
                                                                   int tri) {
  extern __shared__ __align__(16) double sy[];
  int64_t ti, tj;  // tile (ti, tj) covers rows s0 + 64 ti .., columns s0 + 64 tj ..
  if (!tri) {
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
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int wm = (w >> 1) * 32, wn = (w & 1) * 32;
  const int g = lane >> 2, t4 = lane & 3;
  double acc[4][4][2];
#pragma unroll
  for (int m = 0; m < 4; ++m)
#pragma unroll
    for (int n = 0; n < 4; ++n) acc[m][n][0] = acc[m][n][1] = 0.0;
  const int nst = (nb + kSyK - 1) / kSyK;
  auto bufA = [&](int s) { return sy + (s & 1) * 2 * kNB * kSyLd; };
  auto bufB = [&](int s) { return sy + (s & 1) * 2 * kNB * kSyLd + kNB * kSyLd; };
  syrk_stage<CH>(H, ldh, M, r0, c0, j0, min(kSyK, nb), bufA(0), bufB(0));
  cp_async_commit();
  for (int s = 0; s < nst; ++s) {
    if (s + 1 < nst) {
      syrk_stage<CH>(H, ldh, M, r0, c0, j0 + (int64_t)(s + 1) * kSyK, min(kSyK, nb - (s + 1) * kSyK), bufA(s + 1),
                     bufB(s + 1));
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const double* A = bufA(s) + (wm + g) * kSyLd + t4;
    const double* B = bufB(s) + (wn + g) * kSyLd + t4;
#pragma unroll
    for (int ks = 0; ks < kSyK; ks += 4) {
      double a[4], b[4];
#pragma unroll
      for (int m = 0; m < 4; ++m) a[m] = A[m * 8 * kSyLd + ks];
#pragma unroll
      for (int n = 0; n < 4; ++n) b[n] = B[n * 8 * kSyLd + ks];
#pragma unroll
      for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int n = 0; n < 4; ++n) dmma_8x8x4(acc[m][n][0], acc[m][n][1], a[m], b[n]);
    }
    __syncthreads();  // the buffer is refilled by the stage after next
  }
#pragma unroll
  for (int m = 0; m < 4; ++m)
#pragma unroll
    for (int n = 0; n < 4; ++n)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int64_t i = r0 + wm + m * 8 + g, j = c0 + wn + n * 8 + 2 * t4 + h;
        if (i < M && j < c_end && j <= i) H[i * ldh + j] -= acc[m][n][h];
      }
}

// The triangular solves of rb_chol_solve apply the diagonal blocks' inverses
// X (kept by rb_cholesky in each block's strict upper triangle):
// mode 0: y = X v (solves L_kk y = v), mode 1: y = X^T v (solves L_kk^T y = v).
// y = X v (mode 0) or X^T v (mode 1) of diagonal block k0 into shared memory,
// by all 256 threads of the block: the block's 64 x 64 entries are staged in
// shared memory first (whole rows, coalesced), then a quad sums each output
// from there in a fixed order; v is read from src[k0 ..]
__device__ __forceinline__ void tri_block_apply(const double* __restrict__ L, int64_t ldh, int64_t k0, int nb,
                                                const double* __restrict__ src, int mode, double* v, double* y,
                                                double (*Xs)[kNB + 1]) {
  const int tid = threadIdx.x;
#pragma unroll 4
  for (int e = tid; e < kNB * kNB; e += 256) {
    const int r = e / kNB, c = e % kNB;
    Xs[r][c] = (r < nb && c < nb) ? L[(k0 + r) * ldh + k0 + c] : 0.0;
  }
  if (tid < nb) v[tid] = src[k0 + tid];
  __syncthreads();
  const int i = tid >> 2, q = tid & 3;
  double s = 0.0;
  if (i < nb) {
    if (mode == 0) {  // X[i][t], t < i, sits at (t, i)
      for (int t = q; t <= i; t += 4) s = fma(t == i ? 1.0 / Xs[i][i] : Xs[t][i], v[t], s);
    } else {  // X[t][i], t > i, sits at (i, t)
      for (int t = i + q; t < nb; t += 4) s = fma(t == i ? 1.0 / Xs[i][i] : Xs[i][t], v[t], s);
    }
  }
  s += __shfl_xor_sync(0xffffffffu, s, 1);
  s += __shfl_xor_sync(0xffffffffu, s, 2);
  if (i < nb && q == 0) y[i] = s;
  __syncthreads();
}

// One forward step of L y = b, fused: every block solves diagonal block k0
// (y = X v, v = x[k0 ..]) itself, block 0 stores y in w, and each block
// subtracts L[r][k0 ..] y from its kSolveRows rows r below the block (rows
// split over the 8 warps; lane c sums columns c and c + 32, then a warp sum
// per row).
constexpr int kSolveRows = 32;
__global__ void __launch_bounds__(256) fwd_solve_kernel(const double* __restrict__ L, int64_t ldh, int64_t M,
                                                        int64_t k0, int nb, double* __restrict__ x,
                                                        double* __restrict__ w) {
  __shared__ double v[kNB], y[kNB];
  __shared__ double Xs[kNB][kNB + 1];
  tri_block_apply(L, ldh, k0, nb, x, 0, v, y, Xs);
  if (blockIdx.x == 0 && threadIdx.x < nb) w[k0 + threadIdx.x] = y[threadIdx.x];
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  constexpr int RW = kSolveRows / 8;  // rows per warp
  const int64_t rb = k0 + nb + blockIdx.x * (int64_t)kSolveRows + wp * RW;
  const double y0 = lane < nb ? y[lane] : 0.0, y1 = lane + 32 < nb ? y[lane + 32] : 0.0;
  double s[RW];
#pragma unroll
  for (int u = 0; u < RW; ++u) {
    const int64_t r = rb + u;
    s[u] = 0.0;
    if (r < M) {
      const double* Lr = L + r * ldh + k0;
      if (lane < nb) s[u] = Lr[lane] * y0;
      if (lane + 32 < nb) s[u] = fma(Lr[lane + 32], y1, s[u]);
    }
  }
#pragma unroll
  for (int u = 0; u < RW; ++u) {
    const double t = warp_sum(s[u]);
    if (lane == 0 && rb + u < M) x[rb + u] -= t;
  }
}

// One backward step of L^T x = y, fused: every block solves diagonal block
// k0 (v = w[k0 ..], the forward solution less the later blocks' terms),
// block 0 stores the result in x, and each block subtracts L[k0 + r][j] y[r]
// from its 32 columns j < k0 of w (8 warps over the block's rows, summed in
// a fixed order).
__global__ void __launch_bounds__(256) bwd_solve_kernel(const double* __restrict__ L, int64_t ldh, int64_t k0, int nb,
                                                        double* __restrict__ w, double* __restrict__ x) {
  __shared__ double v[kNB], y[kNB], part[8][32];
  __shared__ double Xs[kNB][kNB + 1];
  tri_block_apply(L, ldh, k0, nb, w, 1, v, y, Xs);
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

// four consecutive entries of a row as FP32 (BF16 widened exactly)
__device__ __forceinline__ float4 ld4f(const float* p) { return __ldcs(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ float4 ld4f(const __nv_bfloat16* p) {
  const uint2 x = __ldcs(reinterpret_cast<const uint2*>(p));
  const __nv_bfloat162 a = *reinterpret_cast<const __nv_bfloat162*>(&x.x);
  const __nv_bfloat162 b = *reinterpret_cast<const __nv_bfloat162*>(&x.y);
  return make_float4(__bfloat162float(a.x), __bfloat162float(a.y), __bfloat162float(b.x), __bfloat162float(b.y));
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

// out[m] = alpha sum_k J[m][k] x[k] + beta out[m] in two passes.  Block
// (cx, ry) takes the 1024 columns [1024 cx, 1024 cx + 1024) (4 per thread,
// one vector load per row) of kGemvNRows rows, so a warp reads whole 512-byte
// row segments and the block's rows stream side by side; each row's block
// sum (fixed-order warp and block reduction) goes to part[m][cx], and
// gemv_n_sum_kernel adds a row's parts (lane-strided, then a warp sum).
// The result is the same bits on every run.
constexpr int kGemvNRows = 16;
constexpr int kGemvNCols = 1024;
template <typename JT>
__global__ void __launch_bounds__(256) gemv_n_part_kernel(const JT* __restrict__ J, int64_t M, int64_t K, int64_t ldj,
                                                          const double* __restrict__ x, double* __restrict__ part,
                                                          int64_t nchunk) {
  __shared__ double red[kGemvNRows][8];
  const int64_t k = (int64_t)blockIdx.x * kGemvNCols + 4 * threadIdx.x;
  const int64_t m0 = (int64_t)blockIdx.y * kGemvNRows;
  double xv[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) xv[j] = (k + j < K) ? x[k + j] : 0.0;
  // every row's load is issued before the first product
  float4 v[kGemvNRows];
#pragma unroll
  for (int r = 0; r < kGemvNRows; ++r)
    v[r] = (k < K && m0 + r < M) ? ld4f(J + (m0 + r) * ldj + k) : make_float4(0.f, 0.f, 0.f, 0.f);
  if (k + 3 >= K) {  // the padded row's entries past K are dropped (they may hold anything)
#pragma unroll
    for (int r = 0; r < kGemvNRows; ++r) {
      if (k + 1 >= K) v[r].y = 0.f;
      if (k + 2 >= K) v[r].z = 0.f;
      if (k + 3 >= K) v[r].w = 0.f;
    }
  }
  double s[kGemvNRows];
#pragma unroll
  for (int r = 0; r < kGemvNRows; ++r) {
    s[r] = fma((double)v[r].x, xv[0], 0.0);
    s[r] = fma((double)v[r].y, xv[1], s[r]);
    s[r] = fma((double)v[r].z, xv[2], s[r]);
    s[r] = fma((double)v[r].w, xv[3], s[r]);
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
#pragma unroll
    for (int q = 0; q < 8; ++q) t += red[threadIdx.x][q];
    part[(m0 + threadIdx.x) * nchunk + blockIdx.x] = t;
  }
}

// a warp per row: out[m] = alpha sum_c part[m][c] + beta out[m]
__global__ void gemv_n_sum_kernel(const double* __restrict__ part, int64_t nchunk, int64_t M, double alpha,
                                  double beta, double* __restrict__ out) {
  const int64_t m = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5);
  if (m >= M) return;
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  for (int64_t c = lane; c < nchunk; c += 32) s += part[m * nchunk + c];
  s = warp_sum(s);
  if (lane == 0) out[m] = alpha * s + (beta != 0.0 ? beta * out[m] : 0.0);
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
template <typename JT, bool VEC>
__global__ void row_sumsq_kernel(const JT* __restrict__ J, int64_t M, int64_t K, int64_t ldj,
                                 double* __restrict__ out, __nv_bfloat16* __restrict__ bf, int64_t ldb) {
  __shared__ double red[32];
  for (int64_t m = blockIdx.x; m < M; m += gridDim.x) {
    double s = 0.0;
    int64_t kpad = K;  // first column of the BF16 row's zero padding
    if constexpr (VEC) {
      // 4 columns per thread and chunk: one 16-byte (BF16: 8-byte) load and
      // one 8-byte store; four chunks' loads are issued before their sums
      kpad = (K + 3) / 4 * 4;
      constexpr int U = 4;
      const int64_t step = 4 * (int64_t)blockDim.x;
      for (int64_t k0 = 4 * (int64_t)threadIdx.x; k0 < K; k0 += U * step) {
        float4 v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int64_t k = k0 + u * step;
          v[u] = k < K ? ld4f(J + m * ldj + k) : make_float4(0.f, 0.f, 0.f, 0.f);  // inside the row (ldj % 4 == 0)
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int64_t k = k0 + u * step;
          if (k >= K) break;
          if (k + 1 >= K) v[u].y = 0.f;  // entries past K are dropped
          if (k + 2 >= K) v[u].z = 0.f;
          if (k + 3 >= K) v[u].w = 0.f;
          s = fma((double)v[u].x, (double)v[u].x, s);
          s = fma((double)v[u].y, (double)v[u].y, s);
          s = fma((double)v[u].z, (double)v[u].z, s);
          s = fma((double)v[u].w, (double)v[u].w, s);
          if (bf) {
            __nv_bfloat162 lo = __floats2bfloat162_rn(v[u].x, v[u].y), hi = __floats2bfloat162_rn(v[u].z, v[u].w);
            uint2 w;
            w.x = *reinterpret_cast<uint32_t*>(&lo);
            w.y = *reinterpret_cast<uint32_t*>(&hi);
            *reinterpret_cast<uint2*>(bf + m * ldb + k) = w;
          }
        }
      }
    } else {
      for (int64_t k = threadIdx.x; k < K; k += blockDim.x) {
        const double v = jval(J[m * ldj + k]);
        s = fma(v, v, s);
        if (bf) bf[m * ldb + k] = __float2bfloat16_rn((float)v);
      }
    }
    if (bf)
      for (int64_t k = kpad + threadIdx.x; k < ldb; k += blockDim.x) bf[m * ldb + k] = __float2bfloat16_rn(0.f);
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

// The two streams of rb_cholesky's look-ahead, per device, created once:
// the panel stream at the device's highest priority, the bulk-update stream
// at the default one; both non-blocking.
struct CholStreams {
  cudaStream_t panel = nullptr, rest = nullptr;
};
static int chol_streams(CholStreams* out) {
  static std::mutex mu;
  static CholStreams per_dev[64];
  int dev = 0;
  RB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(RB_ESIZE, "rb_cholesky: device index %d out of range", dev);
  std::lock_guard<std::mutex> lock(mu);
  CholStreams& c = per_dev[dev];
  if (!c.panel) {
    int least = 0, greatest = 0;
    RB_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    RB_CUDA_TRY(cudaStreamCreateWithPriority(&c.panel, cudaStreamNonBlocking, greatest));
    RB_CUDA_TRY(cudaStreamCreateWithPriority(&c.rest, cudaStreamNonBlocking, least));
  }
  *out = c;
  return RB_OK;
}

// events without timing, destroyed with the set
struct EventSet {
  cudaEvent_t e[4] = {nullptr, nullptr, nullptr, nullptr};
  int n = 0;
  int make(int k) {
    for (; n < k; ++n) RB_CUDA_TRY(cudaEventCreateWithFlags(&e[n], cudaEventDisableTiming));
    return RB_OK;
  }
  ~EventSet() {
    for (int i = 0; i < n; ++i) cudaEventDestroy(e[i]);
  }
};

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
  // 16-byte panel copies when every row of H starts on a 16-byte boundary
  const bool ch16 = (reinterpret_cast<uintptr_t>(H) % 16 == 0) && (ldh % 2 == 0);
  auto syrk = ch16 ? syrk_update_kernel<16> : syrk_update_kernel<8>;
  RB_CUDA_TRY(cudaFuncSetAttribute(syrk, cudaFuncAttributeMaxDynamicSharedMemorySize, kSyrkSmem));
  // Right-looking in outer blocks of kOuter columns: inside a block each
  // 64-wide panel is factored (diagonal block, panel solve) and updates only
  // the rest of the block's columns; the trailing matrix then takes one
  // update of depth kOuter per outer block.  Look-ahead: that update is
  // split into the next block's column band (on the panel stream, so the
  // next block can start at once) and the rest of the trailing triangle (on
  // a second stream, overlapping the next block's serial panel work).  The
  // panel stream has the higher priority, so its small launches take SMs as
  // the bulk update's CTAs retire.  Ordering: the rest update of block b
  // waits for block b's panels (event ev_p); the band update of block b + 1,
  // which writes tiles the rest update of block b also writes, waits for it
  // (event ev_r).  Both streams fork from and join back into the caller's.
  CholStreams cs;
  RB_TRY(chol_streams(&cs));
  cudaStream_t sp = cs.panel, sr = cs.rest;
  EventSet ev;
  RB_TRY(ev.make(4));
  cudaEvent_t ev_in = ev.e[0], ev_p = ev.e[1], ev_r = ev.e[2], ev_out = ev.e[3];
  RB_CUDA_TRY(cudaEventRecord(ev_in, st));
  RB_CUDA_TRY(cudaStreamWaitEvent(sp, ev_in, 0));
  RB_CUDA_TRY(cudaStreamWaitEvent(sr, ev_in, 0));
  bool rest_queued = false;
  constexpr int64_t kOuter = 4 * kNB;
  for (int64_t J0 = 0; J0 < M; J0 += kOuter) {
    const int64_t bend = std::min<int64_t>(J0 + kOuter, M);
    for (int64_t j0 = J0; j0 < bend; j0 += kNB) {
      const int nb = (int)std::min<int64_t>(kNB, M - j0);
      potrf_diag_kernel<<<1, 256, 0, sp>>>(H, ldh, j0, nb, err);
      RB_LAUNCH_CHECK();
      const int64_t rest = M - j0 - nb;
      if (rest <= 0) break;
      trsm_panel_kernel<<<(unsigned)ceil_div(rest, kNB), 256, kTrsmSmem, sp>>>(H, ldh, M, j0, nb);
      RB_LAUNCH_CHECK();
      if (j0 + nb < bend) {  // the block's later panels
        const int64_t T = ceil_div(rest, kNB), Tc = ceil_div(bend - (j0 + nb), kNB);
        syrk<<<dim3((unsigned)T, (unsigned)Tc), kSyrkThreads, kSyrkSmem, sp>>>(H, ldh, M, j0, nb, j0 + nb, bend, 0);
        RB_LAUNCH_CHECK();
      }
    }
    const int64_t rest = M - bend;
    if (rest <= 0) break;
    const int depth = (int)(bend - J0);
    const int64_t band_end = std::min<int64_t>(bend + kOuter, M);
    RB_CUDA_TRY(cudaEventRecord(ev_p, sp));  // block J0's panels are final
    if (rest_queued) RB_CUDA_TRY(cudaStreamWaitEvent(sp, ev_r, 0));
    {  // the next block's columns [bend, band_end), all rows below bend
      const int64_t T = ceil_div(rest, kNB), Tc = ceil_div(band_end - bend, kNB);
      syrk<<<dim3((unsigned)T, (unsigned)Tc), kSyrkThreads, kSyrkSmem, sp>>>(H, ldh, M, J0, depth, bend, band_end,
                                                                              0);
      RB_LAUNCH_CHECK();
    }
    if (band_end < M) {  // the trailing triangle right of the band
      const int64_t T = ceil_div(M - band_end, kNB);
      RB_CUDA_TRY(cudaStreamWaitEvent(sr, ev_p, 0));
      syrk<<<(unsigned)(T * (T + 1) / 2), kSyrkThreads, kSyrkSmem, sr>>>(H, ldh, M, J0, depth, band_end, M, 1);
      RB_LAUNCH_CHECK();
      RB_CUDA_TRY(cudaEventRecord(ev_r, sr));
      rest_queued = true;
    }
  }
  RB_CUDA_TRY(cudaEventRecord(ev_out, sr));
  RB_CUDA_TRY(cudaStreamWaitEvent(st, ev_out, 0));
  RB_CUDA_TRY(cudaEventRecord(ev_out, sp));
  RB_CUDA_TRY(cudaStreamWaitEvent(st, ev_out, 0));
  int herr = 0;
  RB_CUDA_TRY(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  RB_CUDA_TRY(cudaStreamSynchronize(st));
  if (herr) return fail(RB_ENOTSPD, "rb_cholesky: non-positive pivot at row %d", herr - 1);
  return RB_OK;
}

size_t rb_chol_solve_work_bytes(int64_t M) { return (size_t)std::max<int64_t>(M, 1) * sizeof(double); }

int rb_chol_solve(const double* L, int64_t M, int64_t ldh, double* x, void* work, size_t work_bytes, void* stream) {
  if (!L || !x || !work || M < 1 || ldh < M) return fail(RB_EARG, "rb_chol_solve: bad arguments");
  if (work_bytes < rb_chol_solve_work_bytes(M)) return fail(RB_EARG, "rb_chol_solve: workspace too small");
  cudaStream_t st = as_stream(stream);
  // one launch per diagonal block and direction: each block of a launch
  // solves the 64 x 64 diagonal step itself and then its share of the update
  double* w = reinterpret_cast<double*>(work);  // the forward solution, consumed by the backward steps
  for (int64_t k0 = 0; k0 < M; k0 += kNB) {  // L y = b
    const int nb = (int)std::min<int64_t>(kNB, M - k0);
    const int64_t rest = M - k0 - nb;
    fwd_solve_kernel<<<(unsigned)std::max<int64_t>(1, ceil_div(rest, kSolveRows)), 256, 0, st>>>(L, ldh, M, k0, nb,
                                                                                                 x, w);
    RB_LAUNCH_CHECK();
  }
  for (int64_t k0 = ((M - 1) / kNB) * kNB; k0 >= 0; k0 -= kNB) {  // L^T x = y
    const int nb = (int)std::min<int64_t>(kNB, M - k0);
    bwd_solve_kernel<<<(unsigned)std::max<int64_t>(1, ceil_div(k0, 32)), 256, 0, st>>>(L, ldh, k0, nb, w, x);
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
                      double* out, void* work, size_t work_bytes, void* stream) {
  if (!J || !x || !out || M < 1 || K < 1 || ldj < K) return fail(RB_EARG, "rb_gemv_n: bad arguments");
  if ((reinterpret_cast<uintptr_t>(J) & (4 * sizeof(JT) - 1)) || (ldj % 4) || ldj < ceil_div(K, 4) * 4)
    return fail(RB_EARG, "rb_gemv_n: J rows must start on %d-byte boundaries and hold K rounded up to 4 entries",
                (int)(4 * sizeof(JT)));
  if (ceil_div(M, kGemvNRows) > 65535) return fail(RB_ESIZE, "rb_gemv_n: too many rows");
  if (!work || work_bytes < rb_gemv_n_work_bytes(M, K)) return fail(RB_EARG, "rb_gemv_n: workspace too small");
  cudaStream_t st = as_stream(stream);
  const int64_t nchunk = ceil_div(K, kGemvNCols);
  double* part = reinterpret_cast<double*>(work);  // M x nchunk row parts
  gemv_n_part_kernel<JT><<<dim3((unsigned)nchunk, (unsigned)ceil_div(M, kGemvNRows)), 256, 0, st>>>(J, M, K, ldj, x,
                                                                                                   part, nchunk);
  RB_LAUNCH_CHECK();
  gemv_n_sum_kernel<<<(unsigned)ceil_div(M, 8), 256, 0, st>>>(part, nchunk, M, alpha, beta, out);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

extern "C" {

size_t rb_gemv_n_work_bytes(int64_t M, int64_t K) {
  return (size_t)std::max<int64_t>(M, 1) * (size_t)std::max<int64_t>(ceil_div(K, kGemvNCols), 1) * sizeof(double);
}

int rb_gemv_n(const float* J, int64_t M, int64_t K, int64_t ldj, const double* x, double alpha, double beta,
              double* out, void* work, size_t work_bytes, void* stream) {
  return gemv_n_run(J, M, K, ldj, x, alpha, beta, out, work, work_bytes, stream);
}

int rb_gemv_n_bf16(const void* J, int64_t M, int64_t K, int64_t ldj, const double* x, double alpha, double beta,
                   double* out, void* work, size_t work_bytes, void* stream) {
  return gemv_n_run(reinterpret_cast<const __nv_bfloat16*>(J), M, K, ldj, x, alpha, beta, out, work, work_bytes,
                    stream);
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
  // vector path: rows start on 4-entry boundaries (and, for the copy, the BF16 rows on 8-byte ones)
  const bool vec = (reinterpret_cast<uintptr_t>(J) % (4 * sizeof(JT)) == 0) && ldj % 4 == 0 &&
                   (!bf || reinterpret_cast<uintptr_t>(bf) % 8 == 0);
  if (vec)
    row_sumsq_kernel<JT, true><<<nb, 256, 0, st>>>(J, M, K, ldj, rows, bf, ldb);
  else
    row_sumsq_kernel<JT, false><<<nb, 256, 0, st>>>(J, M, K, ldj, rows, bf, ldb);
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
