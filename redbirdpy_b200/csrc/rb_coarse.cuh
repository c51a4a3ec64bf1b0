// Coarse-space correction of the Krylov preconditioner (included by rb_krylov.cu).
//
// The rows (mesh nodes) are grouped into nc aggregates (the caller bins the
// nodes by position).  With P the n x nc 0/1 matrix of the grouping, the
// preconditioner is
//     z = D^-1 r + P X P^T r,      X = (P^T A P)^-1   (nc x nc, dense)
// i.e. Jacobi plus an exact solve on the aggregated operator: the
// smooth error that Jacobi-CG removes slowly is removed by the coarse solve.
// P^T A P is summed from the CSR values in a fixed order and inverted once per
// solve by blocked Gauss-Jordan in FP64 (no pivoting: the aggregated FEM
// operator is symmetric positive definite, or complex symmetric with a
// positive definite real part); each application is a restriction (one read
// of r), one nc x nc x k product and the prolongation folded into the
// p-update.  The r.z dot product needed by CG splits the same way:
//     r.z = sum_i r_i d_i r_i + sum_I (P^T r)_I (X P^T r)_I .
#pragma once

#include <type_traits>

namespace rb {

constexpr int kCoarseMax = 4096;  // largest aggregate count (one row of P^T A P in shared memory)
constexpr int kGjB = 64;          // Gauss-Jordan block
constexpr int kCoarseSplits = 8;  // most K splits of the X rc product

// ------------------------------------------------------------------ GEMM
// C_z = alpha AT^T B + beta C (row-major; AT is kk x m, B is kk x n, so both
// operand tiles load along rows and land in shared memory untransposed; beta
// == 0 does not read C).  The coarse product passes X itself as AT (X is
// symmetric: the inverse of the symmetric aggregated operator); Gauss-Jordan
// passes the block column transposed.  64 x BN tiles, 16-deep k steps, 256
// threads with 4 x BN/16 outputs each; the next k step's tiles are fetched
// into registers while the current one is used.  Split K: block z takes the
// k range [z kchunk, (z + 1) kchunk) and writes C + z cstride.  SCALE false:
// C = AT^T B with a plain store (the coarse product; measured 0.054 against
// 0.0625 ms per iteration with the scaled epilogue).
template <typename T, int BN, bool SCALE>
__global__ void __launch_bounds__(256) gemm_tn_kernel(int64_t m, int64_t n, int64_t kk, T alpha,
                                                      const T* __restrict__ AT, int64_t lda, const T* __restrict__ B,
                                                      int64_t ldb, T beta, int beta_zero, T* __restrict__ C,
                                                      int64_t ldc, int64_t kchunk, int64_t cstride,
                                                      const int32_t* __restrict__ live) {
  if (live && *live == 0) return;  // inside the Krylov loop: every column converged
  constexpr int BM = 64, BK = 16, TM = 4, TN = BN / 16;
  constexpr int LA = BM * BK / 256, LB = BN * BK / 256;  // tile elements each thread loads
  __shared__ __align__(16) T As[BK][BM];
  __shared__ __align__(16) T Bs[BK][BN];
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;  // output columns tx*TN.., rows ty*TM..
  const int64_t r0 = (int64_t)blockIdx.y * BM, c0 = (int64_t)blockIdx.x * BN;
  const int64_t kb = (int64_t)blockIdx.z * kchunk, ke = std::min<int64_t>(kk, kb + kchunk);
  C += (int64_t)blockIdx.z * cstride;
  T acc[TM][TN];
#pragma unroll
  for (int u = 0; u < TM; ++u)
#pragma unroll
    for (int v = 0; v < TN; ++v) acc[u][v] = s_zero(T());
  T ra[LA], rb[LB];
  auto fetch = [&](int64_t k0) {
#pragma unroll
    for (int l = 0; l < LA; ++l) {
      const int e = tid + 256 * l, q = e / BM, i = e % BM;
      ra[l] = (k0 + q < ke && r0 + i < m) ? AT[(k0 + q) * lda + r0 + i] : s_zero(T());
    }
#pragma unroll
    for (int l = 0; l < LB; ++l) {
      const int e = tid + 256 * l, q = e / BN, j = e % BN;
      rb[l] = (k0 + q < ke && c0 + j < n) ? B[(k0 + q) * ldb + c0 + j] : s_zero(T());
    }
  };
  if (kb < ke) fetch(kb);
  for (int64_t k0 = kb; k0 < ke; k0 += BK) {
#pragma unroll
    for (int l = 0; l < LA; ++l) {
      const int e = tid + 256 * l;
      As[e / BM][e % BM] = ra[l];
    }
#pragma unroll
    for (int l = 0; l < LB; ++l) {
      const int e = tid + 256 * l;
      Bs[e / BN][e % BN] = rb[l];
    }
    __syncthreads();
    if (k0 + BK < ke) fetch(k0 + BK);
#pragma unroll
    for (int q = 0; q < BK; ++q) {
      T a[TM], b[TN];
#pragma unroll
      for (int u = 0; u < TM; ++u) a[u] = As[q][ty * TM + u];
#pragma unroll
      for (int v = 0; v < TN; ++v) b[v] = Bs[q][tx * TN + v];
#pragma unroll
      for (int u = 0; u < TM; ++u)
#pragma unroll
        for (int v = 0; v < TN; ++v) acc[u][v] = s_fma(a[u], b[v], acc[u][v]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < TM; ++u)
#pragma unroll
    for (int v = 0; v < TN; ++v) {
      const int64_t i = r0 + ty * TM + u, j = c0 + tx * TN + v;
      if (i < m && j < n) {
        if constexpr (SCALE) {
          T x = s_mul(alpha, acc[u][v]);
          if (!beta_zero) x = s_fma(beta, C[i * ldc + j], x);
          C[i * ldc + j] = x;
        } else {
          C[i * ldc + j] = acc[u][v];
        }
      }
    }
}

// 64 x 64 tiles (79 registers for FP32, three blocks per SM): coarse product
// and dot 54 us per iteration at nc = 2048, k = 128 against 67 us with 64 x 128
// tiles (127 registers, two blocks per SM); complex128 takes 64 x 32 tiles
template <typename T> constexpr int gemm_bn() { return sizeof(T) >= 16 ? 32 : 64; }

template <typename T> static T h_real(double v);
static bool h_is_one(float a) { return a == 1.0f; }
static bool h_is_one(double a) { return a == 1.0; }
static bool h_is_one(cfloat a) { return a.x == 1.0f && a.y == 0.0f; }
static bool h_is_one(cdouble a) { return a.x == 1.0 && a.y == 0.0; }

template <typename T>
static int gemm_tn(int64_t m, int64_t n, int64_t kk, T alpha, const T* AT, int64_t lda, const T* B, int64_t ldb,
                   T beta, bool beta_zero, T* C, int64_t ldc, cudaStream_t st, int splits = 1, int64_t cstride = 0,
                   const int32_t* live = nullptr) {
  if (m <= 0 || n <= 0) return RB_OK;
  constexpr int BN = gemm_bn<T>();
  const int64_t kchunk = ceil_div(ceil_div(kk, splits), 16) * 16;
  dim3 g((unsigned)ceil_div(n, BN), (unsigned)ceil_div(m, 64), (unsigned)splits);
  const bool plain = beta_zero && h_is_one(alpha);
  if (plain)
    gemm_tn_kernel<T, BN, false><<<g, 256, 0, st>>>(m, n, kk, alpha, AT, lda, B, ldb, beta, 1, C, ldc, kchunk,
                                                   cstride, live);
  else
    gemm_tn_kernel<T, BN, true><<<g, 256, 0, st>>>(m, n, kk, alpha, AT, lda, B, ldb, beta, beta_zero ? 1 : 0, C, ldc,
                                                  kchunk, cstride, live);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

__device__ __forceinline__ double s_inv(double a) { return 1.0 / a; }
__device__ __forceinline__ cdouble s_inv(cdouble a) {
  const double d = a.x * a.x + a.y * a.y;
  return make_double2(a.x / d, -a.y / d);
}
__device__ __forceinline__ bool s_bad(double a) { return !(a != 0.0) || !isfinite(a); }
__device__ __forceinline__ bool s_bad(cdouble a) {
  return (a.x == 0.0 && a.y == 0.0) || !isfinite(a.x) || !isfinite(a.y);
}
__device__ __forceinline__ double s_neg(double a) { return -a; }
__device__ __forceinline__ cdouble s_neg(cdouble a) { return make_double2(-a.x, -a.y); }

// ------------------------------------------- Gauss-Jordan on one 64-block
// Dinv = (A[b0.., b0..])^-1 for the nb x nb diagonal block.  Two copies of
// the block in shared memory: pivot step c reads one and writes the other
// (one barrier per pivot).  Thread t owns column t % 64 of rows t / 64 + 4 u.
constexpr int kGjLd = kGjB + 1;
template <typename T>
constexpr size_t gj_smem_bytes() { return sizeof(T) * 2 * kGjB * kGjLd; }

template <typename T>
__global__ void __launch_bounds__(256) gj_diag_kernel(const T* __restrict__ A, int64_t lda, int64_t b0, int nb,
                                                      T* __restrict__ Dinv, int* __restrict__ err) {
  extern __shared__ __align__(16) unsigned char gsm[];
  T* cur = reinterpret_cast<T*>(gsm);
  T* nxt = cur + kGjB * kGjLd;
  const int tid = threadIdx.x;
  const int j = tid & (kGjB - 1), ib = tid / kGjB;
#pragma unroll
  for (int u = 0; u < kGjB / 4; ++u) {
    const int i = ib + 4 * u;
    cur[i * kGjLd + j] = (i < nb && j < nb) ? A[(b0 + i) * lda + b0 + j] : s_zero(T());
  }
  __syncthreads();
  for (int c = 0; c < nb; ++c) {
    const T piv = cur[c * kGjLd + c];
    if (s_bad(piv)) {  // uniform: every thread reads the same pivot
      if (tid == 0) atomicExch(err, 1);
      return;
    }
    const T ip = s_inv(piv);
    const T rcj = s_mul(cur[c * kGjLd + j], ip);  // scaled pivot row
#pragma unroll
    for (int u = 0; u < kGjB / 4; ++u) {
      const int i = ib + 4 * u;
      const T mic = cur[i * kGjLd + c];
      T v;
      if (i == c) v = (j == c) ? ip : rcj;
      else v = (j == c) ? s_neg(s_mul(mic, ip)) : s_sub(cur[i * kGjLd + j], s_mul(mic, rcj));
      nxt[i * kGjLd + j] = v;
    }
    __syncthreads();
    T* t = cur;
    cur = nxt;
    nxt = t;
  }
#pragma unroll
  for (int u = 0; u < kGjB / 4; ++u) {
    const int i = ib + 4 * u;
    Dinv[i * kGjB + j] = (i < nb && j < nb) ? cur[i * kGjLd + j] : s_zero(T());
  }
}

// CbT[j][i] = A[i][b0 + j], the block column transposed (rows of the block
// itself zero); kGjB x nc, ld nc
template <typename T>
__global__ void gj_cols_kernel(const T* __restrict__ A, int64_t nc, int64_t b0, int nb, T* __restrict__ CbT) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nc * kGjB;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int j = (int)(e / nc);
    const int64_t i = e % nc;
    CbT[e] = (j < nb && (i < b0 || i >= b0 + nb)) ? A[i * nc + b0 + j] : s_zero(T());
  }
}

// A[b0 + i][:] = R[i][:]  and  A[b0 + i][b0 + j] = Dinv[i][j]
template <typename T>
__global__ void gj_rows_kernel(T* __restrict__ A, int64_t nc, int64_t b0, int nb, const T* __restrict__ R,
                               const T* __restrict__ Dinv) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)nb * nc;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / nc, j = e % nc;
    A[(b0 + i) * nc + j] = (j >= b0 && j < b0 + nb) ? Dinv[i * kGjB + (j - b0)] : R[e];
  }
}

// ---------------------------------------------------- P^T A P (dense)
// one warp per aggregate I: row I of P^T A P in shared memory; the lane that
// owns coarse column J (J % 32) adds every entry of that column in the order
// of the aggregate's rows and their CSR entries (deterministic)
template <typename T64>
__global__ void __launch_bounds__(32) coarse_build_kernel(int64_t nc, const int32_t* __restrict__ indptr,
                                                          const int32_t* __restrict__ indices,
                                                          const T64* __restrict__ val,
                                                          const int32_t* __restrict__ agg,
                                                          const int32_t* __restrict__ agg_ptr,
                                                          const int32_t* __restrict__ agg_rows, T64* __restrict__ Ac) {
  extern __shared__ __align__(16) unsigned char csm[];
  T64* row = reinterpret_cast<T64*>(csm);
  const int lane = threadIdx.x;
  const int64_t I = blockIdx.x;
  for (int64_t j = lane; j < nc; j += 32) row[j] = s_zero(T64());
  __syncwarp();
  const int32_t q0 = agg_ptr[I], q1 = agg_ptr[I + 1];
  for (int32_t qb = q0; qb < q1; qb += 32) {
    // the bounds of the next 32 rows, one per lane
    const int nr = min(32, q1 - qb);
    int32_t mb = 0, me = 0;
    if (lane < nr) {
      const int32_t i = agg_rows[qb + lane];
      mb = indptr[i];
      me = indptr[i + 1];
    }
    for (int r = 0; r < nr; ++r) {
      const int32_t b = __shfl_sync(0xffffffffu, mb, r), e = __shfl_sync(0xffffffffu, me, r);
      for (int32_t p0 = b; p0 < e; p0 += 32) {
        const int cnt = min(32, e - p0);
        int32_t J = -1;
        T64 v = s_zero(T64());
        if (lane < cnt) {
          J = agg[indices[p0 + lane]];
          v = val[p0 + lane];
        }
        for (int u = 0; u < cnt; ++u) {
          const int32_t Ju = __shfl_sync(0xffffffffu, J, u);
          const T64 vu = shfl_s(v, u);
          if ((Ju & 31) == lane) row[Ju] = s_add(row[Ju], vu);
        }
      }
    }
  }
  __syncwarp();
  for (int64_t j = lane; j < nc; j += 32) Ac[I * nc + j] = row[j];
}

template <typename T64, typename T>
__global__ void cast_kernel(int64_t count, const T64* __restrict__ a, T* __restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
    if constexpr (Scalar<T>::is_complex) {
      b[i] = T{(typename Scalar<T>::real)a[i].x, (typename Scalar<T>::real)a[i].y};
    } else {
      b[i] = (T)a[i];
    }
  }
}

// ------------------------------------------------------ per application
// rc[I][c] = sum over the rows i of aggregate I of r[i][c] (accumulated in
// the acc type): one block per aggregate; warp w takes the aggregate's rows
// w*32 .. w*32+31, w*32+256 .. (4 row fetches in flight), lanes over columns
// lane + 32 t; the 8 warps' sums are added in warp order
template <typename T>
__global__ void __launch_bounds__(256) restrict_kernel(int64_t nc, int64_t k, const T* __restrict__ R,
                                                       const int32_t* __restrict__ agg_ptr,
                                                       const int32_t* __restrict__ agg_rows, T* __restrict__ rc,
                                                       const int32_t* __restrict__ live) {
  if (live && *live == 0) return;  // inside the Krylov loop: every column converged
  typedef typename Scalar<T>::acc A;
  __shared__ A red[8][128];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int64_t I = blockIdx.x; I < nc; I += gridDim.x) {
    A s[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) s[t] = acc_zero<A>();
    const int32_t q0 = agg_ptr[I], q1 = agg_ptr[I + 1];
    for (int32_t qb = q0 + 32 * w; qb < q1; qb += 256) {
      const int cnt = min(32, q1 - qb);
      const int32_t my = lane < cnt ? agg_rows[qb + lane] : 0;
      for (int j = 0; j < cnt; j += 4) {
        T v[4][4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int32_t row = __shfl_sync(0xffffffffu, my, min(j + u, cnt - 1));
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            const int64_t c = lane + 32 * t;
            v[u][t] = (c < k && j + u < cnt) ? R[(int64_t)row * k + c] : s_zero(T());
          }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int t = 0; t < 4; ++t) s[t] = acc_add(s[t], to_acc(v[u][t]));
      }
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) red[w][lane + 32 * t] = s[t];
    __syncthreads();
    for (int c = threadIdx.x; c < k; c += 256) {
      A t = acc_zero<A>();
#pragma unroll
      for (int q = 0; q < 8; ++q) t = acc_add(t, red[q][c]);
      if constexpr (Scalar<T>::is_complex) {
        rc[I * k + c] = T{(typename Scalar<T>::real)t.x, (typename Scalar<T>::real)t.y};
      } else {
        rc[I * k + c] = (T)t;
      }
    }
    __syncthreads();
  }
}

// ec[I][c] = sum over the splits s (in order) of es[s][I][c];
// part[block][c] = sum over this block's aggregates of rc[I][c] ec[I][c] (unconjugated)
constexpr int kCdotGrid = 256;  // one aggregate per warp at nc = 2048
template <typename T>
__global__ void __launch_bounds__(256) coarse_dot_kernel(int64_t nc, int64_t k, const T* __restrict__ rc,
                                                         const T* __restrict__ es, int splits,
                                                         T* __restrict__ ec,
                                                         typename Scalar<T>::acc* __restrict__ part,
                                                         const int32_t* __restrict__ live) {
  if (live && *live == 0) return;  // inside the Krylov loop: every column converged
  typedef typename Scalar<T>::acc A;
  __shared__ A red[8][128];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  A s[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) s[u] = acc_zero<A>();
  for (int64_t I = blockIdx.x * 8 + w; I < nc; I += (int64_t)gridDim.x * 8) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int64_t c = lane + 32 * u;
      if (c < k) {
        T e = es[I * k + c];
        for (int q = 1; q < splits; ++q) e = s_add(e, es[(int64_t)q * nc * k + I * k + c]);
        ec[I * k + c] = e;
        s[u] = acc_fma(rc[I * k + c], e, s[u]);
      }
    }
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) red[w][lane + 32 * u] = s[u];
  __syncthreads();
  for (int c = threadIdx.x; c < k; c += 256) {
    A t = acc_zero<A>();
    for (int q = 0; q < 8; ++q) t = acc_add(t, red[q][c]);
    part[(int64_t)blockIdx.x * k + c] = t;
  }
}

// ------------------------------------------------------------- host side
template <typename T> static T h_real(double v);
template <> float h_real<float>(double v) { return (float)v; }
template <> double h_real<double>(double v) { return v; }
template <> cfloat h_real<cfloat>(double v) { return make_float2((float)v, 0.f); }
template <> cdouble h_real<cdouble>(double v) { return make_double2(v, 0.0); }

// what one application needs
template <typename T>
struct CoarseOp {
  int64_t nc = 0;
  const int32_t *agg = nullptr, *agg_ptr = nullptr, *agg_rows = nullptr;
  T *X = nullptr, *rc = nullptr, *ec = nullptr;
  T* es = nullptr;       // split-K partial products, kCoarseSplits x nc x k
  void* part = nullptr;  // kCdotGrid x k acc
};

// setup buffers (FP64) besides the operator itself
template <typename T64, typename T>
struct CoarseBufs {
  CoarseOp<T> op;
  T64 *A64 = nullptr, *Rb = nullptr, *Cb = nullptr, *Dinv = nullptr;  // Cb: the block column, transposed
  int* err = nullptr;
};

template <typename T64, typename T, typename Cv>
static size_t coarse_carve(Cv& cv, CoarseBufs<T64, T>& c, int64_t nc, int64_t k) {
  c.op.nc = nc;
  c.A64 = cv.template take<T64>(nc * nc);
  c.Rb = cv.template take<T64>(kGjB * nc);
  c.Cb = cv.template take<T64>(nc * kGjB);
  c.Dinv = cv.template take<T64>(kGjB * kGjB);
  c.op.X = cv.template take<T>(nc * nc);
  c.op.rc = cv.template take<T>(nc * k);
  c.op.ec = cv.template take<T>(nc * k);
  c.op.es = cv.template take<T>((size_t)kCoarseSplits * nc * k);
  c.op.part = cv.template take<cdouble>((size_t)kCdotGrid * k);
  c.err = cv.template take<int>(1);
  return cv.used;
}

// X = (P^T A P)^-1 from the FP64 values of A
template <typename T64, typename T>
static int coarse_setup(const rb_csr& A, CoarseBufs<T64, T>& c, cudaStream_t st) {
  const int64_t nc = c.op.nc;
  const size_t rowb = (size_t)nc * sizeof(T64);
  RB_CUDA_TRY(cudaFuncSetAttribute(coarse_build_kernel<T64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rowb));
  coarse_build_kernel<T64><<<(unsigned)nc, 32, rowb, st>>>(nc, A.indptr, A.indices, (const T64*)A.val64, c.op.agg,
                                                           c.op.agg_ptr, c.op.agg_rows, c.A64);
  RB_LAUNCH_CHECK();
  RB_CUDA_TRY(cudaMemsetAsync(c.err, 0, sizeof(int), st));
  const T64 one = h_real<T64>(1.0), mone = h_real<T64>(-1.0), zero = h_real<T64>(0.0);
  const unsigned eg = (unsigned)std::min<int64_t>(ceil_div(nc * kGjB, 256), 148 * 8);
  constexpr size_t gj_smem = gj_smem_bytes<T64>();
  RB_CUDA_TRY(cudaFuncSetAttribute(gj_diag_kernel<T64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gj_smem));
  for (int64_t b0 = 0; b0 < nc; b0 += kGjB) {
    const int nb = (int)std::min<int64_t>(kGjB, nc - b0);
    gj_diag_kernel<T64><<<1, 256, gj_smem, st>>>(c.A64, nc, b0, nb, c.Dinv, c.err);
    RB_LAUNCH_CHECK();
    // R = Dinv A[b, :]  (Dinv is symmetric: the inverse of a diagonal block
    // of the symmetric Schur complement, so it serves as its own transpose)
    RB_TRY(gemm_tn<T64>(nb, nc, nb, one, c.Dinv, kGjB, c.A64 + b0 * nc, nc, zero, true, c.Rb, nc, st));
    // CbT = (A[:, b])^T with the block's own rows zeroed
    gj_cols_kernel<T64><<<eg, 256, 0, st>>>(c.A64, nc, b0, nb, c.Cb);
    RB_LAUNCH_CHECK();
    // A -= Cb R (rank-nb update of every row outside the block)
    RB_TRY(gemm_tn<T64>(nc, nc, nb, mone, c.Cb, nc, c.Rb, nc, one, false, c.A64, nc, st));
    // A[:, b] = -Cb Dinv outside the block; A[b, :] = R; A[b, b] = Dinv
    RB_TRY(gemm_tn<T64>(nc, nb, nb, mone, c.Cb, nc, c.Dinv, kGjB, zero, true, c.A64 + b0, nc, st));
    gj_rows_kernel<T64><<<eg, 256, 0, st>>>(c.A64, nc, b0, nb, c.Rb, c.Dinv);
    RB_LAUNCH_CHECK();
  }
  cast_kernel<T64, T><<<(unsigned)std::min<int64_t>(ceil_div(nc * nc, 256), 148 * 16), 256, 0, st>>>(nc * nc, c.A64,
                                                                                                     c.op.X);
  RB_LAUNCH_CHECK();
  int herr = 0;
  RB_CUDA_TRY(cudaMemcpyAsync(&herr, c.err, sizeof(int), cudaMemcpyDeviceToHost, st));
  RB_CUDA_TRY(cudaStreamSynchronize(st));
  if (herr) return fail(RB_EBREAKDOWN, "rb_femsolve: the aggregated operator has a zero or non-finite pivot");
  return RB_OK;
}

// rc = P^T r (unless R is NULL: rc already holds it), ec = X rc,
// part = column sums of rc * ec; live as the Krylov loop's kernels
template <typename T>
static int coarse_apply(const CoarseOp<T>& c, const T* R, int64_t k, cudaStream_t st,
                        const int32_t* live = nullptr) {
  const int64_t nc = c.nc;
  if (R) {
    restrict_kernel<T><<<(unsigned)std::min<int64_t>(nc, 148 * 16), 256, 0, st>>>(nc, k, R, c.agg_ptr, c.agg_rows,
                                                                                  c.rc, live);
    RB_LAUNCH_CHECK();
  }
  // enough blocks for two per SM: split the nc-long sums (fixed order, no atomics)
  const T one = h_real<T>(1.0), zero = h_real<T>(0.0);
  const int64_t tiles = ceil_div(nc, 64) * ceil_div(k, gemm_bn<T>());
  const int splits = (int)std::max<int64_t>(1, std::min<int64_t>({kCoarseSplits, ceil_div(2 * 148, tiles),
                                                                   ceil_div(nc, 256)}));
  RB_TRY(gemm_tn<T>(nc, k, nc, one, c.X, nc, c.rc, k, zero, true, c.es, k, st, splits, nc * k, live));
  coarse_dot_kernel<T><<<kCdotGrid, 256, 0, st>>>(nc, k, c.rc, c.es, splits, c.ec, (typename Scalar<T>::acc*)c.part,
                                                  live);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

}  // namespace rb
