// Multi-RHS sparse solve: CSR SpMM with fused column reductions, Jacobi-
// preconditioned block CG (real SPD) / block COCG (complex symmetric) on all
// right-hand sides at once, wrapped in FP64 iterative refinement.
//
// Layout: every n x k multi-vector is row-major (column index fastest).  A
// group of L lanes owns one row at a time; lane l owns the V consecutive
// columns [l*V, l*V+V) for the whole kernel, so per-column dot products are
// accumulated per lane (in FP64) and reduced once per block into a
// [grid x k] partials array.  A one-block "finalize" kernel then reduces the
// partials in fixed order and updates the per-column CG scalars on the
// device; the host only polls a counter of active columns every few
// iterations.  Columns are frozen individually when they converge.
#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "rb_common.cuh"

namespace rb {

constexpr int kBlk = 256;
// resident blocks per SM of the row kernels, by scalar type: sets both the
// register budget (__launch_bounds__) and the single-wave grid size
template <typename T> struct Bps { static constexpr int value = 4; };
// complex128 vector kernels: 2 blocks (128 registers); at 3 the CG update
// spilled 300 B (row order) and 476 B (aggregate order)
template <> struct Bps<cdouble> { static constexpr int value = 2; };
// complex64 vector kernels: 3 blocks (85 registers); at 4 the CG update
// spilled (88 B in row order, 272 B in aggregate order)
template <> struct Bps<cfloat> { static constexpr int value = 3; };
// SpMM: 4 blocks per SM for the FP32 types (8 gathers in flight need the
// registers; measured best), 3 for complex128 (no spills in the residual form)
template <typename T> struct BpsSpmm { static constexpr int value = Bps<T>::value; };
template <> struct BpsSpmm<cfloat> { static constexpr int value = 4; };
template <> struct BpsSpmm<cdouble> { static constexpr int value = 3; };
constexpr int kGridMax = 148 * 8;       // upper bound of any grid (partials arrays)

// ----------------------------------------------------------- vector access
template <typename T, int V>
__device__ __forceinline__ void ldv(const T* __restrict__ p, T (&o)[V]) {
  constexpr int B = V * (int)sizeof(T);
  if constexpr (B % 16 == 0) {
    const int4* q = reinterpret_cast<const int4*>(p);
    int4* d = reinterpret_cast<int4*>(o);
#pragma unroll
    for (int j = 0; j < B / 16; ++j) d[j] = __ldg(q + j);
  } else if constexpr (B % 8 == 0) {
    const int2* q = reinterpret_cast<const int2*>(p);
    int2* d = reinterpret_cast<int2*>(o);
#pragma unroll
    for (int j = 0; j < B / 8; ++j) d[j] = __ldg(q + j);
  } else {
#pragma unroll
    for (int j = 0; j < V; ++j) o[j] = p[j];
  }
}
template <typename T, int V>
__device__ __forceinline__ void ldv_s(const T* p, T (&o)[V]) {  // shared memory
  constexpr int B = V * (int)sizeof(T);
  if constexpr (B % 16 == 0) {
    const int4* q = reinterpret_cast<const int4*>(p);
    int4* d = reinterpret_cast<int4*>(o);
#pragma unroll
    for (int j = 0; j < B / 16; ++j) d[j] = q[j];
  } else if constexpr (B % 8 == 0) {
    const int2* q = reinterpret_cast<const int2*>(p);
    int2* d = reinterpret_cast<int2*>(o);
#pragma unroll
    for (int j = 0; j < B / 8; ++j) d[j] = q[j];
  } else {
#pragma unroll
    for (int j = 0; j < V; ++j) o[j] = p[j];
  }
}
template <typename T, int V>
__device__ __forceinline__ void stv(T* __restrict__ p, const T (&o)[V]) {
  constexpr int B = V * (int)sizeof(T);
  if constexpr (B % 16 == 0) {
    int4* q = reinterpret_cast<int4*>(p);
    const int4* d = reinterpret_cast<const int4*>(o);
#pragma unroll
    for (int j = 0; j < B / 16; ++j) q[j] = d[j];
  } else if constexpr (B % 8 == 0) {
    int2* q = reinterpret_cast<int2*>(p);
    const int2* d = reinterpret_cast<const int2*>(o);
#pragma unroll
    for (int j = 0; j < B / 8; ++j) q[j] = d[j];
  } else {
#pragma unroll
    for (int j = 0; j < V; ++j) p[j] = o[j];
  }
}

// Rows are dealt to the groups of all blocks in interleaved order: at any
// moment the whole grid works inside one window of consecutive rows, so the
// x rows that matrix rows i and i +- (layer size) share are still in L2 when
// the second one needs them.

template <typename A> __device__ __forceinline__ A acc_zero();
template <> __device__ __forceinline__ double acc_zero<double>() { return 0.0; }
template <> __device__ __forceinline__ cdouble acc_zero<cdouble>() { return make_double2(0.0, 0.0); }
__device__ __forceinline__ double acc_add(double a, double b) { return a + b; }
__device__ __forceinline__ cdouble acc_add(cdouble a, cdouble b) { return make_double2(a.x + b.x, a.y + b.y); }

// Block-reduce per-lane column accumulators acc[V] (lane l owns columns
// l*V..) into part[blockIdx.x * k + c].
// With S column slices, group g of the block owns slice g % S.
template <typename A, int L, int V, int S = 1>
__device__ __forceinline__ void block_colreduce(const A (&acc)[V], A* __restrict__ part, int64_t k,
                                                A* sm /* kBlk * V */) {
  const int lane = threadIdx.x % L, grp = threadIdx.x / L;
  constexpr int G = kBlk / L;
#pragma unroll
  for (int j = 0; j < V; ++j) sm[(grp * L + lane) * V + j] = acc[j];
  __syncthreads();
  for (int c = threadIdx.x; c < S * L * V; c += kBlk) {
    if (c < k) {
      const int sl = c / (L * V), l = (c % (L * V)) / V, j = c % V;
      A s = acc_zero<A>();
      for (int g = sl; g < G; g += S) s = acc_add(s, sm[(g * L + l) * V + j]);
      part[(int64_t)blockIdx.x * k + c] = s;
    }
  }
  __syncthreads();
}

__device__ __forceinline__ float shfl_s(float v, int l) { return __shfl_sync(0xffffffffu, v, l); }
__device__ __forceinline__ double shfl_s(double v, int l) { return __shfl_sync(0xffffffffu, v, l); }
__device__ __forceinline__ cfloat shfl_s(cfloat v, int l) {
  return make_float2(__shfl_sync(0xffffffffu, v.x, l), __shfl_sync(0xffffffffu, v.y, l));
}
__device__ __forceinline__ cdouble shfl_s(cdouble v, int l) {
  return make_double2(__shfl_sync(0xffffffffu, v.x, l), __shfl_sync(0xffffffffu, v.y, l));
}

// ------------------------------------------------------------------ SpMM
// Epilogues after y = (A x)[row, cols]:
enum { EPI_STORE = 0, EPI_PQDOT = 1, EPI_RESID = 2 };

// y_row = A_row x; EPI_STORE: Y = y; EPI_PQDOT: Y = y, acc += x_row*y (unconj);
// EPI_RESID: Y = B - y, acc += |B - y|^2   (B real FP64)
// S column slices (S = 1, or 2 for complex64 at 128 columns): a lane group
// takes (row, slice) tasks, slice = task % S, so that a lane keeps 16 bytes
// per gathered row and 8 gathers in flight; the group count is a multiple of
// S, so a group always sees the same slice (and its column sums stay put).
// O32: n k < 2^31, so that the staged x row offsets (index k, in elements)
// fit an int32 and a gather address is one wide multiply-add
template <typename T, int L, int V, int EPI, int S = 1, bool O32 = true>
__global__ void __launch_bounds__(kBlk, BpsSpmm<T>::value)
spmm_kernel(int64_t n, int64_t k, const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
            const T* __restrict__ val, const T* __restrict__ X, T* __restrict__ Y,
            const double* __restrict__ B, void* __restrict__ part_, const int32_t* __restrict__ live) {
  if (live && *live == 0) return;  // every column converged: a no-op iteration
  // residual norms accumulate |r|^2 in double; dot products in the acc type
  typedef std::conditional_t<EPI == EPI_RESID, double, typename Scalar<T>::acc> A;
  A* part = reinterpret_cast<A*>(part_);
  __shared__ A sm[(EPI == EPI_STORE) ? 1 : kBlk * V];
  __shared__ __align__(16) int32_t s_off[L == 32 ? kBlk : 1];  // per-warp (x row offset or index, value) chunks
  __shared__ __align__(16) T s_val[L == 32 ? kBlk : 1];
  // what a chunk entry holds: the x row offset index * k (O32), else the index
  auto staged = [&](int32_t idx) -> int32_t { return O32 ? idx * (int32_t)k : idx; };
  const int lane = threadIdx.x % L;
  const int64_t task0 = blockIdx.x * (int64_t)(kBlk / L) + threadIdx.x / L;
  const int64_t c0 = (task0 % S) * (int64_t)(L * V) + (int64_t)lane * V;
  const bool on = c0 < k;
  const int64_t groups = (int64_t)gridDim.x * (kBlk / L);
  alignas(16) A acc[V];
#pragma unroll
  for (int j = 0; j < V; ++j) acc[j] = acc_zero<A>();
  // FP32 rows are software-pipelined: the bounds of the row two tasks ahead
  // and the first (index, value) chunk of the next row are loaded while the
  // current row's gathers run, so that a row's first gathers do not wait for
  // the indptr -> indices chain (0.287 -> 0.265 ms at 128 columns on the
  // 520k-node box; the sliced complex64 form measured slower with it, 0.61 ->
  // 0.71 ms, and keeps the plain loop)
  constexpr bool PIPE = (L == 32) && std::is_same<T, float>::value;
  constexpr int U = (V * sizeof(T) <= 16) ? 8 : 4;
  const int64_t ntask = n * S;
  auto chunk0 = [&](int32_t bb, int32_t ee, int32_t& oo, T& vv) {
    const int c = min(32, ee - bb);
    const int cp = (c + U - 1) / U * U;
    oo = 0;
    vv = s_zero(T());
    if (lane < cp) {
      oo = staged(indices[bb + min(lane, c - 1)]);
      if (lane < c) vv = val[bb + lane];
    }
  };
  int32_t pb0 = 0, pe0 = 0, pb1 = 0, pe1 = 0, ci = 0;
  T cv = s_zero(T());
  if constexpr (PIPE) {
    if (task0 < ntask) {
      pb0 = indptr[task0 / S];
      pe0 = indptr[task0 / S + 1];
    }
    if (task0 + groups < ntask) {
      pb1 = indptr[(task0 + groups) / S];
      pe1 = indptr[(task0 + groups) / S + 1];
    }
    chunk0(pb0, pe0, ci, cv);
  }
  for (int64_t task = task0; task < ntask; task += groups) {
    const int64_t row = task / S;
    int32_t b, e;
    if constexpr (PIPE) {
      b = pb0;
      e = pe0;
    } else {
      b = indptr[row];
      e = indptr[row + 1];
    }
    alignas(16) T y[V];
#pragma unroll
    for (int j = 0; j < V; ++j) y[j] = s_zero(T());
    if constexpr (L == 32) {
      // whole warp on one row: lanes fetch a chunk of the row's indices and
      // values once (coalesced) into the warp's shared-memory slot, the index
      // already turned into the element offset of its x row, and every lane
      // then reads U of them at a time with 16-byte broadcast loads and
      // gathers from its own base pointer with one wide multiply-add.  (Broadcasting by
      // shuffle cost two L1 data-pipe wavefronts per nonzero, ~30% of that
      // pipe, the SpMM's binding unit; the index arithmetic per gather was
      // most of the issued instructions.)  The chunk is padded to a multiple
      // of U with copies of its last index at coefficient 0 (same NaN
      // behaviour as the exact product) rather than falling back to one
      // dependent load at a time.
      int32_t* const wo = s_off + (threadIdx.x & ~31);
      T* const wv = s_val + (threadIdx.x & ~31);
      const T* const xl = X + c0;  // this lane's columns of x row 0
      int32_t pb2 = 0, pe2 = 0, ni = 0;
      T nv = s_zero(T());
      if constexpr (PIPE) {
        const int64_t t2 = task + 2 * groups;
        if (t2 < ntask) {
          pb2 = indptr[t2 / S];
          pe2 = indptr[t2 / S + 1];
        }
        chunk0(pb1, pe1, ni, nv);
      }
      for (int32_t p0 = b; p0 < e; p0 += 32) {
        const int cnt = min(32, e - p0);
        const int cntp = (cnt + U - 1) / U * U;
        if (PIPE && p0 == b) {
          if (lane < cntp) {
            wo[lane] = ci;
            wv[lane] = cv;
          }
        } else if (lane < cntp) {
          wo[lane] = staged(indices[p0 + min(lane, cnt - 1)]);
          wv[lane] = (lane < cnt) ? val[p0 + lane] : s_zero(T());
        }
        __syncwarp();
        for (int j = 0; j < cntp; j += U) {
          alignas(16) int32_t oo[U];
          alignas(16) T aa[U];
          ldv_s<int32_t, U>(wo + j, oo);
          ldv_s<T, U>(wv + j, aa);
          if (on) {
            alignas(16) T xv[U][V];
#pragma unroll
            for (int u = 0; u < U; ++u) {
              const T* src = O32 ? xl + (uint32_t)oo[u] : xl + (int64_t)oo[u] * k;
              ldv<T, V>(src, xv[u]);
            }
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
              for (int q = 0; q < V; ++q) y[q] = s_fma(aa[u], xv[u][q], y[q]);
          }
        }
        __syncwarp();  // the slot is rewritten by the next chunk
      }
      if constexpr (PIPE) {
        pb0 = pb1;
        pe0 = pe1;
        pb1 = pb2;
        pe1 = pe2;
        ci = ni;
        cv = nv;
      }
    } else if (on) {
#pragma unroll 4
      for (int32_t p = b; p < e; ++p) {
        const T a = val[p];
        alignas(16) T xv[V];
        ldv<T, V>(X + (int64_t)indices[p] * k + c0, xv);
#pragma unroll
        for (int j = 0; j < V; ++j) y[j] = s_fma(a, xv[j], y[j]);
      }
    }
    if (on) {
      if constexpr (EPI == EPI_RESID) {
        alignas(16) double bv[V];
#pragma unroll
        for (int j = 0; j < V; ++j) bv[j] = B[row * k + c0 + j];
#pragma unroll
        for (int j = 0; j < V; ++j) {
          T r = y[j];
          if constexpr (Scalar<T>::is_complex) {
            r.x = (typename Scalar<T>::real)bv[j] - r.x;
            r.y = -r.y;
          } else {
            r = (T)bv[j] - r;
          }
          y[j] = r;
          acc[j] += s_abs2(r);
        }
      }
      if constexpr (EPI == EPI_PQDOT) {
        alignas(16) T xv[V];
        ldv<T, V>(X + row * k + c0, xv);
#pragma unroll
        for (int j = 0; j < V; ++j) {
          if constexpr (EPI == EPI_PQDOT) acc[j] = acc_fma(xv[j], y[j], acc[j]);
        }
      }
      stv<T, V>(Y + row * k + c0, y);
    }
  }
  if (EPI != EPI_STORE) block_colreduce<A, L, V, S>(acc, part, k, sm);
}

// ------------------------------------------------ row-group SpMM (k = 32 V)
// Rows are taken G consecutive at a time.  The union of the G rows' column
// lists (ascending, each with a G-bit mask of the rows holding that column)
// is built once per solve.  A warp walks its groups' unions: each union
// column's x row (k values, 16-byte aligned) is fetched ONCE for the whole
// group by a bulk copy (cp.async.bulk, completion counted on an mbarrier)
// into a two-chunk ring in the warp's shared memory, and every row of the
// group that holds the column takes its FMAs from there.  Lane l owns columns
// [l V, l V + V).  On a tetrahedral mesh numbered with locality (a structured
// box: x fastest) 8 consecutive rows need ~70 x rows instead of 8 x 15, and
// the fetches of one union run over consecutive rows of x.
// Used for the FP64 Krylov types (1-2 KB rows at 128 columns), where it
// measured 12% (double) and 29% (complex128) faster than spmm_kernel on the
// 3M-tet box; for FP32 rows (512 B) spmm_kernel's register gathers are faster
// (0.31 ms vs 0.57 ms per launch) and stay in use.
template <typename T> struct GrpCfg {
  static constexpr bool enabled = sizeof(T) >= 8 && !std::is_same<T, cfloat>::value;
  static constexpr int G = 4;  // rows per group
  static constexpr int C = 4096 / (32 * 4 * (int)sizeof(T)) > 0 ? 4096 / (32 * 4 * (int)sizeof(T)) : 1;
};
template <> struct GrpCfg<float> {
  static constexpr bool enabled = false;  // FP32 takes the row-pair SpMM below
  static constexpr int G = 2;             // rows per group of its union plan
  static constexpr int C = 8;
};
template <> struct GrpCfg<cfloat> {
  static constexpr bool enabled = false;  // complex64 takes the row-pair SpMM below
  static constexpr int G = 2;
  static constexpr int C = 8;
};
// Row-pair SpMM: FP32 at 65..128 columns (multiples of 4: L = 32, V = 4);
// complex64 at 128 columns in two 64-column slices (V = 2, S = 2)
template <typename T> struct PairCfg {
  static constexpr bool enabled = std::is_same<T, float>::value || std::is_same<T, cfloat>::value;
  static constexpr int V = std::is_same<T, float>::value ? 4 : 2;
  static constexpr int S = std::is_same<T, float>::value ? 1 : 2;
};
template <typename T> static bool pair_cols_ok(int64_t k) {
  if (std::is_same<T, float>::value) return k > 64 && k <= 128 && k % 4 == 0;
  return k == 128;
}
constexpr int kGrpWarps = 4;     // warps per block
constexpr int kGrpVals = 256;    // staged matrix values per group (else read from global)
constexpr int kWaitSpins = 1 << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// bounded wait for the phase with the given parity to complete
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (int i = 0; i < kWaitSpins; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
    if (i > 64) __nanosleep(32);
  }
  return false;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// union sizes (count pass) or union entries (fill pass) of each row group
template <int G, bool FILL>
__global__ void group_union_kernel(int64_t n, const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
                                   int32_t* __restrict__ cnt_or_ptr, int32_t* __restrict__ ucol,
                                   uint8_t* __restrict__ umask) {
  const int64_t ng = (n + G - 1) / G;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < ng; g += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r0 = g * G;
    int32_t p[G], e[G];
#pragma unroll
    for (int r = 0; r < G; ++r) {
      const bool in = r0 + r < n;
      p[r] = in ? indptr[r0 + r] : 0;
      e[r] = in ? indptr[r0 + r + 1] : 0;
    }
    int32_t c = 0, out = FILL ? cnt_or_ptr[g] : 0;
    while (true) {
      int32_t m = 0x7fffffff;
#pragma unroll
      for (int r = 0; r < G; ++r)
        if (p[r] < e[r]) m = min(m, indices[p[r]]);
      if (m == 0x7fffffff) break;
      uint32_t mask = 0;
#pragma unroll
      for (int r = 0; r < G; ++r)
        if (p[r] < e[r] && indices[p[r]] == m) {
          mask |= 1u << r;
          ++p[r];
        }
      if (FILL) {
        ucol[out + c] = m;
        umask[out + c] = (uint8_t)mask;
      }
      ++c;
    }
    if (!FILL) cnt_or_ptr[g] = c;
  }
}

struct GroupPlan {
  const int32_t* gptr;  // ng + 1
  const int32_t* ucol;
  const uint8_t* umask;
  int64_t ng;
};

// Y rows of one group, with the epilogues of spmm_kernel
template <typename T, int V, int EPI, typename A>
__device__ __forceinline__ void grp_epilogue(int64_t row, int64_t k, int64_t c0, T (&y)[V], const T* __restrict__ X,
                                             T* __restrict__ Y, const double* __restrict__ B, A (&acc)[V]) {
  if constexpr (EPI == EPI_RESID) {
#pragma unroll
    for (int j = 0; j < V; ++j) {
      const double bv = B[row * k + c0 + j];
      T r = y[j];
      if constexpr (Scalar<T>::is_complex) {
        r.x = (typename Scalar<T>::real)bv - r.x;
        r.y = -r.y;
      } else {
        r = (T)bv - r;
      }
      y[j] = r;
      acc[j] += s_abs2(r);
    }
  }
  if constexpr (EPI == EPI_PQDOT) {
    alignas(16) T xv[V];
    ldv<T, V>(X + row * k + c0, xv);
#pragma unroll
    for (int j = 0; j < V; ++j) acc[j] = acc_fma(xv[j], y[j], acc[j]);
  }
  stv<T, V>(Y + row * k + c0, y);
}

template <typename T, int V, int EPI>
__global__ void __launch_bounds__(kGrpWarps * 32)
spmm_grp_kernel(int64_t n, const int32_t* __restrict__ indptr, const T* __restrict__ val, GroupPlan gp,
                const T* __restrict__ X, T* __restrict__ Y, const double* __restrict__ B, void* __restrict__ part_,
                int32_t* __restrict__ err, const int32_t* __restrict__ live) {
  if (live && *live == 0) return;  // every column converged: a no-op iteration
  constexpr int G = GrpCfg<T>::G, C = GrpCfg<T>::C;
  constexpr int64_t k = 32 * V;
  constexpr uint32_t rowbytes = (uint32_t)(k * sizeof(T));
  typedef std::conditional_t<EPI == EPI_RESID, double, typename Scalar<T>::acc> A;
  extern __shared__ __align__(128) unsigned char dsm[];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // per-warp carve: [2 C rows of x][kGrpVals values][2 mbarriers]
  constexpr size_t warp_bytes = (size_t)2 * C * rowbytes + (size_t)kGrpVals * sizeof(T) + 16;
  unsigned char* base = dsm + wid * warp_bytes;
  T* ring = reinterpret_cast<T*>(base);
  T* sval = reinterpret_cast<T*>(base + (size_t)2 * C * rowbytes);
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + (size_t)2 * C * rowbytes + (size_t)kGrpVals * sizeof(T));
  if (lane == 0) {
    mbar_init(bar, 1);
    mbar_init(bar + 1, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  const int64_t c0 = (int64_t)lane * V;
  const int64_t W = (int64_t)gridDim.x * kGrpWarps;
  const int64_t w = (int64_t)blockIdx.x * kGrpWarps + wid;
  const int64_t ng = gp.ng;

  // producer cursor over the warp's chunks (groups w, w + W, ...; empty
  // unions are skipped, chunks never span two groups)
  int64_t pg = w;
  int32_t pu = 0, pue = 0;
  if (pg < ng) { pu = gp.gptr[pg]; pue = gp.gptr[pg + 1]; }
  auto advance = [&]() {
    while (pu >= pue && pg < ng) {
      pg += W;
      if (pg < ng) { pu = gp.gptr[pg]; pue = gp.gptr[pg + 1]; }
    }
  };
  uint32_t m0 = 0, m1 = 0;  // lane j: row mask of entry j of the chunk in buffer 0 / 1
  bool pend0 = false, pend1 = false;
  auto issue = [&](int buf) {
    advance();
    if (pg >= ng) return;
    const int cnt = min(C, pue - pu);
    int32_t col = 0;
    uint32_t msk = 0;
    if (lane < cnt) {
      col = gp.ucol[pu + lane];
      msk = gp.umask[pu + lane];
    }
    if (lane == 0) mbar_expect_tx(bar + buf, (uint32_t)cnt * rowbytes);
    __syncwarp();
    // order the warp's reads of this buffer before the copies that overwrite it
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (lane < cnt) bulk_g2s(ring + (size_t)(buf * C + lane) * k, X + (int64_t)col * k, rowbytes, bar + buf);
    if (buf) { m1 = msk; pend1 = true; } else { m0 = msk; pend0 = true; }
    pu += cnt;
  };
  issue(0);
  issue(1);

  alignas(16) A acc[V];
#pragma unroll
  for (int j = 0; j < V; ++j) acc[j] = acc_zero<A>();
  uint32_t ph0 = 0, ph1 = 0;
  int buf = 0;
  bool ok = true;
  for (int64_t g = w; g < ng && ok; g += W) {
    const int64_t r0 = g * G;
    const int nr = (int)((n - r0 < G) ? (n - r0) : G);
    // value offsets of the group's rows (consecutive rows: one value range)
    const int32_t ip = (lane <= nr) ? indptr[r0 + lane] : 0;
    const int32_t vb = __shfl_sync(0xffffffffu, ip, 0);
    const int32_t vt = __shfl_sync(0xffffffffu, ip, nr) - vb;
    int32_t vp[G];
#pragma unroll
    for (int r = 0; r < G; ++r) vp[r] = __shfl_sync(0xffffffffu, ip, r < nr ? r : nr) - vb;
    const bool staged = vt <= kGrpVals;
    if (staged)
      for (int t = lane; t < vt; t += 32) sval[t] = val[vb + t];
    __syncwarp();
    alignas(16) T y[G][V];
#pragma unroll
    for (int r = 0; r < G; ++r)
#pragma unroll
      for (int j = 0; j < V; ++j) y[r][j] = s_zero(T());
    const int32_t ue = gp.gptr[g + 1];
    for (int32_t u = gp.gptr[g]; u < ue; u += C) {
      const int cnt = min(C, ue - u);
      if (!mbar_wait(bar + buf, buf ? ph1 : ph0)) { ok = false; break; }
      if (buf) { ph1 ^= 1; pend1 = false; } else { ph0 ^= 1; pend0 = false; }
      const uint32_t mreg = buf ? m1 : m0;
      const T* xs = ring + (size_t)buf * C * k + c0;
      for (int j = 0; j < cnt; ++j) {
        const uint32_t m = __shfl_sync(0xffffffffu, mreg, j);
        alignas(16) T xv[V];
        ldv_s<T, V>(xs + (size_t)j * k, xv);
#pragma unroll
        for (int r = 0; r < G; ++r) {
          if (m & (1u << r)) {
            const T a = staged ? sval[vp[r]] : val[vb + vp[r]];
            ++vp[r];
#pragma unroll
            for (int q = 0; q < V; ++q) y[r][q] = s_fma(a, xv[q], y[r][q]);
          }
        }
      }
      __syncwarp();
      issue(buf);
      buf ^= 1;
    }
    if (!ok) break;
#pragma unroll
    for (int r = 0; r < G; ++r)
      if (r < nr) grp_epilogue<T, V, EPI, A>(r0 + r, k, c0, y[r], X, Y, B, acc);
    __syncwarp();  // the next group's values overwrite sval
  }
  if (!ok) {
    if (lane == 0) atomicExch(err, 1);
    // let the copies still in flight land before the shared memory goes away
    if (pend0) mbar_wait(bar, ph0);
    if (pend1) mbar_wait(bar + 1, ph1);
  }
  if constexpr (EPI != EPI_STORE) {
    // block partials: warps' lanes own the same columns
    __shared__ A red[kGrpWarps][32 * V];
#pragma unroll
    for (int j = 0; j < V; ++j) red[wid][c0 + j] = acc[j];
    __syncthreads();
    A* part = reinterpret_cast<A*>(part_);
    for (int c = threadIdx.x; c < k; c += kGrpWarps * 32) {
      A s2 = acc_zero<A>();
#pragma unroll
      for (int q = 0; q < kGrpWarps; ++q) s2 = acc_add(s2, red[q][c]);
      part[(int64_t)blockIdx.x * k + c] = s2;
    }
  }
}

template <typename T>
constexpr size_t grp_smem_bytes() {
  return (size_t)kGrpWarps *
         ((size_t)2 * GrpCfg<T>::C * 32 * 4 * sizeof(T) + (size_t)kGrpVals * sizeof(T) + 16);
}

// ----------------------------------------------------- row-pair SpMM (FP32)
// A warp takes rows 2t and 2t+1 together and walks the union of their
// column lists (the group plan with G = 2: ascending columns, each with a
// 2-bit mask of the rows holding it), gathering each x row once and applying
// it to both rows (coefficient 0 where a row lacks the column).  On the
// tetrahedral box the union holds 73% of the two rows' nonzeros, so 27% fewer
// 512-byte gathers go through L1, the per-row kernel's binding unit, for
// twice the FMAs per gather.  A row's coefficients come straight from its
// CSR values: the position of a union entry within row r is the count of
// earlier entries with bit r set (warp ballot + popc, carried across chunks).
// Chunks of 32 union entries are staged in shared memory as (x row offset,
// coefficient of row 0, coefficient of row 1), padded to a multiple of U with
// the last offset at coefficient 0.  EPI as spmm_kernel (PQDOT only here).
// T = complex64: S = 2 column slices of 64; a task is (pair, slice) and a
// warp always sees the same slice (task % S = warp % S, groups a multiple of
// S), as block_colreduce requires.
template <typename T, int EPI>
__global__ void __launch_bounds__(kBlk, BpsSpmm<T>::value)
spmm_pair_kernel(int64_t n, int64_t k, const int32_t* __restrict__ indptr, const T* __restrict__ val, GroupPlan gp,
                 const T* __restrict__ X, T* __restrict__ Y, void* __restrict__ part_,
                 const int32_t* __restrict__ live) {
  if (live && *live == 0) return;  // every column converged: a no-op iteration
  constexpr int V = PairCfg<T>::V, S = PairCfg<T>::S, U = 8;
  typedef typename Scalar<T>::acc A;
  static_assert(EPI == EPI_PQDOT, "row-pair SpMM: p.Ap epilogue only");
  __shared__ A sm[kBlk * V];
  __shared__ __align__(16) int32_t s_off[kBlk];
  __shared__ __align__(16) T s_va[kBlk];
  __shared__ __align__(16) T s_vb[kBlk];
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const int64_t task0 = blockIdx.x * (int64_t)(kBlk / 32) + (threadIdx.x >> 5);
  const int64_t c0 = (task0 % S) * (int64_t)(32 * V) + (int64_t)lane * V;
  const bool on = c0 < k;
  const int64_t groups = (int64_t)gridDim.x * (kBlk / 32);
  int32_t* const wo = s_off + (threadIdx.x & ~31);
  T* const wa = s_va + (threadIdx.x & ~31);
  T* const wb = s_vb + (threadIdx.x & ~31);
  const T* const xl = X + c0;
  alignas(16) A acc[V];
#pragma unroll
  for (int j = 0; j < V; ++j) acc[j] = acc_zero<A>();
  for (int64_t task = task0; task < gp.ng * S; task += groups) {
    const int64_t t = task / S;
    const int64_t r0 = 2 * t;
    const bool has1 = r0 + 1 < n;
    const int32_t ub = gp.gptr[t], ue = gp.gptr[t + 1];
    const int32_t ba = indptr[r0], bb = indptr[r0 + 1];  // value ranges of rows r0 and r0 + 1
    int32_t ca = 0, cb = 0;                              // entries of each row consumed so far
    alignas(16) T ya[V], yb[V];
#pragma unroll
    for (int j = 0; j < V; ++j) ya[j] = yb[j] = s_zero(T());
    for (int32_t u0 = ub; u0 < ue; u0 += 32) {
      const int cnt = min(32, ue - u0);
      const int cntp = (cnt + U - 1) / U * U;
      const bool in = lane < cnt;
      const int32_t col = in ? gp.ucol[u0 + lane] : 0;
      const uint32_t m = in ? gp.umask[u0 + lane] : 0u;
      const unsigned bma = __ballot_sync(0xffffffffu, m & 1u), bmb = __ballot_sync(0xffffffffu, m & 2u);
      const T va = (m & 1u) ? val[ba + ca + __popc(bma & lt)] : s_zero(T());
      const T vb = (m & 2u) ? val[bb + cb + __popc(bmb & lt)] : s_zero(T());
      ca += __popc(bma);
      cb += __popc(bmb);
      const int32_t last = __shfl_sync(0xffffffffu, col, cnt - 1);
      if (lane < cntp) {
        wo[lane] = (in ? col : last) * (int32_t)k;
        wa[lane] = va;
        wb[lane] = vb;
      }
      __syncwarp();
      for (int j = 0; j < cntp; j += U) {
        alignas(16) int32_t oo[U];
        ldv_s<int32_t, U>(wo + j, oo);
        if (on) {
          alignas(16) T xv[U][V];
#pragma unroll
          for (int u = 0; u < U; ++u) ldv<T, V>(xl + (uint32_t)oo[u], xv[u]);
          alignas(16) T aa[U], bbv[U];
          ldv_s<T, U>(wa + j, aa);
          ldv_s<T, U>(wb + j, bbv);
#pragma unroll
          for (int u = 0; u < U; ++u)
#pragma unroll
            for (int q = 0; q < V; ++q) {
              ya[q] = s_fma(aa[u], xv[u][q], ya[q]);
              yb[q] = s_fma(bbv[u], xv[u][q], yb[q]);
            }
        }
      }
      __syncwarp();  // the slot is rewritten by the next chunk
    }
    if (on) {
      alignas(16) T pv[V];
      ldv<T, V>(X + r0 * k + c0, pv);
#pragma unroll
      for (int j = 0; j < V; ++j) acc[j] = acc_fma(pv[j], ya[j], acc[j]);
      stv<T, V>(Y + r0 * k + c0, ya);
      if (has1) {
        ldv<T, V>(X + (r0 + 1) * k + c0, pv);
#pragma unroll
        for (int j = 0; j < V; ++j) acc[j] = acc_fma(pv[j], yb[j], acc[j]);
        stv<T, V>(Y + (r0 + 1) * k + c0, yb);
      }
    }
  }
  block_colreduce<A, 32, V, S>(acc, reinterpret_cast<A*>(part_), k, sm);
}

// ------------------------------------------------------- CG vector kernels
// relres, stagnation and the per-column scale of the next correction
struct OuterState {
  double bnorm;
  double relres;
  double prev;
  double scale;
  double itol2;  // squared inner tolerance of the next sweep
  int32_t active;
  int32_t done;  // 1 converged, 2 stagnated, 3 non-finite residual
};

// Per-column state of the inner Krylov iteration (device).
struct ColState {
  cdouble rz;      // (r, z) unconjugated (real solves use .x)
  cdouble pq;      // (p, A p)
  cdouble alpha;
  cdouble beta;
  double rr;       // ||r||^2
  double rr0;      // ||r_0||^2
  double tol2;     // squared relative tolerance of this column's sweep (< 0: the solve's own)
  int32_t active;  // column still iterating
  int32_t status;  // 0 running/converged, 2 breakdown
  int32_t iters;
  int32_t upd;     // x += alpha p in this iteration's p-update (alpha set by fin_alpha)
};

template <typename T> __device__ __forceinline__ T from_c(cdouble v);
template <> __device__ __forceinline__ float from_c<float>(cdouble v) { return (float)v.x; }
template <> __device__ __forceinline__ double from_c<double>(cdouble v) { return v.x; }
template <> __device__ __forceinline__ cfloat from_c<cfloat>(cdouble v) { return make_float2((float)v.x, (float)v.y); }
template <> __device__ __forceinline__ cdouble from_c<cdouble>(cdouble v) { return v; }
__device__ __forceinline__ cdouble to_c(double v) { return make_double2(v, 0.0); }
__device__ __forceinline__ cdouble to_c(cdouble v) { return v; }

}  // namespace rb

#include "rb_coarse.cuh"

namespace rb {

// init: p = z = Dinv r (+ ec[agg[row]], the coarse correction, when agg is
// given); acc0 += r.p (unconj), acc1 += |r|^2; x = 0
template <typename T, int L, int V>
__global__ void __launch_bounds__(kBlk, Bps<T>::value)
cg_init_kernel(int64_t n, int64_t k, const T* __restrict__ dinv, const T* __restrict__ R, T* __restrict__ P,
               T* __restrict__ Xs, typename Scalar<T>::acc* __restrict__ part_rz, double* __restrict__ part_rr,
               const int32_t* __restrict__ agg, const T* __restrict__ ec) {
  typedef typename Scalar<T>::acc A;
  __shared__ A sm[kBlk * V];
  __shared__ double smr[kBlk * V];
  const int lane = threadIdx.x % L;
  const int64_t c0 = (int64_t)lane * V;
  const bool on = c0 < k;
  const int64_t groups = (int64_t)gridDim.x * (kBlk / L);
  alignas(16) A arz[V];
  alignas(16) double arr[V];
#pragma unroll
  for (int j = 0; j < V; ++j) { arz[j] = acc_zero<A>(); arr[j] = 0.0; }
  for (int64_t row = blockIdx.x * (int64_t)(kBlk / L) + threadIdx.x / L; row < n; row += groups) {
    if (!on) continue;
    const T d = dinv[row];
    alignas(16) T r[V], p[V], z[V], e[V];
    ldv<T, V>(R + row * k + c0, r);
    if (agg) {
      ldv<T, V>(ec + (int64_t)agg[row] * k + c0, e);
    } else {
#pragma unroll
      for (int j = 0; j < V; ++j) e[j] = s_zero(T());
    }
#pragma unroll
    for (int j = 0; j < V; ++j) {
      p[j] = s_fma(d, r[j], e[j]);
      z[j] = s_zero(T());
      arz[j] = acc_fma(r[j], p[j], arz[j]);
      arr[j] += s_abs2(r[j]);
    }
    stv<T, V>(P + row * k + c0, p);
    stv<T, V>(Xs + row * k + c0, z);
  }
  block_colreduce<A, L, V>(arz, part_rz, k, sm);
  block_colreduce<double, L, V>(arr, part_rr, k, smr);
}

// r -= a q; z = Dinv r; acc rz += r.z, rr += |r|^2.  (x += a p waits for
// the p-update, which reads p anyway: 3 vector passes here instead of 6.)
template <typename T, int L, int V>
__global__ void __launch_bounds__(kBlk, Bps<T>::value)
cg_update_kernel(int64_t n, int64_t k, const ColState* __restrict__ cs, const T* __restrict__ dinv,
                 T* __restrict__ R, const T* __restrict__ Q, typename Scalar<T>::acc* __restrict__ part_rz,
                 double* __restrict__ part_rr, const int32_t* __restrict__ live) {
  if (live && *live == 0) return;  // every column converged: a no-op iteration
  typedef typename Scalar<T>::acc A;
  __shared__ A sm[kBlk * V];
  __shared__ double smr[kBlk * V];
  const int lane = threadIdx.x % L;
  const int64_t c0 = (int64_t)lane * V;
  const bool on = c0 < k;
  const int64_t groups = (int64_t)gridDim.x * (kBlk / L);
  alignas(16) T al[V];
  bool act[V];
#pragma unroll
  for (int j = 0; j < V; ++j) {
    act[j] = on && cs[c0 + j].active;
    al[j] = act[j] ? from_c<T>(cs[c0 + j].alpha) : s_zero(T());
  }
  alignas(16) A arz[V];
  alignas(16) double arr[V];
#pragma unroll
  for (int j = 0; j < V; ++j) { arz[j] = acc_zero<A>(); arr[j] = 0.0; }
  for (int64_t row = blockIdx.x * (int64_t)(kBlk / L) + threadIdx.x / L; row < n; row += groups) {
    if (!on) continue;
    const T d = dinv[row];
    alignas(16) T r[V], q[V];
    ldv<T, V>(R + row * k + c0, r);
    ldv<T, V>(Q + row * k + c0, q);
#pragma unroll
    for (int j = 0; j < V; ++j) {
      if (act[j]) r[j] = s_sub(r[j], s_mul(al[j], q[j]));  // frozen columns keep r untouched
      const T z = s_mul(d, r[j]);
      arz[j] = acc_fma(r[j], z, arz[j]);
      arr[j] += s_abs2(r[j]);
    }
    stv<T, V>(R + row * k + c0, r);
  }
  block_colreduce<A, L, V>(arz, part_rz, k, sm);
  block_colreduce<double, L, V>(arr, part_rr, k, smr);
}

// x += alpha p (columns whose alpha this iteration set: cs.upd), then
// p = z + beta p, z = Dinv r (+ ec[agg[row]] with a coarse space) (columns
// still active)
template <typename T, int V>
struct PupCols {
  alignas(16) T al[V], be[V];
  bool act[V], upd[V];
  bool any_act = false, any_upd = false;
  __device__ __forceinline__ void load(const ColState* __restrict__ cs, int64_t c0) {
#pragma unroll
    for (int j = 0; j < V; ++j) {
      act[j] = cs[c0 + j].active;
      upd[j] = cs[c0 + j].upd;
      al[j] = upd[j] ? from_c<T>(cs[c0 + j].alpha) : s_zero(T());
      be[j] = from_c<T>(cs[c0 + j].beta);
      any_act |= act[j];
      any_upd |= upd[j];
    }
  }
  __device__ __forceinline__ void row(T* __restrict__ Xrow, T* __restrict__ Prow, const T* __restrict__ Rrow, T d,
                                      const T (&e)[V]) const {
    alignas(16) T p[V];
    ldv<T, V>(Prow, p);
    if (any_upd) {
      alignas(16) T x[V];
      ldv<T, V>(Xrow, x);
#pragma unroll
      for (int j = 0; j < V; ++j)
        if (upd[j]) x[j] = s_fma(al[j], p[j], x[j]);
      stv<T, V>(Xrow, x);
    }
    if (any_act) {
      alignas(16) T r[V];
      ldv<T, V>(Rrow, r);
#pragma unroll
      for (int j = 0; j < V; ++j)
        if (act[j]) p[j] = s_fma(be[j], p[j], s_fma(d, r[j], e[j]));
      stv<T, V>(Prow, p);
    }
  }
};

template <typename T, int L, int V>
__global__ void __launch_bounds__(kBlk, Bps<T>::value)
cg_pupdate_kernel(int64_t n, int64_t k, const ColState* __restrict__ cs, const T* __restrict__ dinv,
                  const T* __restrict__ R, T* __restrict__ P, T* __restrict__ Xs, const int32_t* __restrict__ agg,
                  const T* __restrict__ ec) {
  const int lane = threadIdx.x % L;
  const int64_t c0 = (int64_t)lane * V;
  if (c0 >= k) return;
  const int64_t groups = (int64_t)gridDim.x * (kBlk / L);
  PupCols<T, V> pc;
  pc.load(cs, c0);
  if (!pc.any_act && !pc.any_upd) return;
  for (int64_t row = blockIdx.x * (int64_t)(kBlk / L) + threadIdx.x / L; row < n; row += groups) {
    const T d = dinv[row];
    alignas(16) T e[V];
    if (agg) {
      ldv<T, V>(ec + (int64_t)agg[row] * k + c0, e);
    } else {
#pragma unroll
      for (int j = 0; j < V; ++j) e[j] = s_zero(T());
    }
    pc.row(Xs + row * k + c0, P + row * k + c0, R + row * k + c0, d, e);
  }
}

// Aggregate-ordered forms of the two kernels above, used with a coarse
// space on real systems: block b takes aggregates b, b + grid, ...; the
// block's lane groups take the aggregate's rows (agg_rows) in turn.  The
// vector updates are row-local, so the order changes no value; what it buys
// is the coarse restriction rc[I] = sum of the aggregate's new r rows, summed
// in registers and then over the groups in fixed order (no extra pass over
// r), and one read of ec[I] per aggregate in the p-update.  Measured on the
// 520k-node box at 128 columns: FP32 update 0.265 ms in either order, 0.12 ms
// less per iteration in all; complex64 update 0.577 ms against 0.525 ms in
// row order, but the coarse step 0.070 ms against 0.285 ms with a separate
// restriction kernel (FD forward 276 ms against 299 ms).  Each lane group
// sums its rows of the aggregate in the vector type (about 30 rows), the
// groups are added in FP64 and the result rounded to the vector type.
template <typename T> struct AggOrder { static constexpr bool value = true; };
// The p-update needs no restriction; it takes the aggregate order only where
// that measured faster: complex64 (214.5 against 217.9 ms for the FD solve);
// FP32 streams better in row order, reading ec[agg[row]] from L2 (CW solve
// 94.2 against 96.6 ms).
template <typename T> struct PupAggOrder { static constexpr bool value = Scalar<T>::is_complex; };
template <typename A, int L, int V, typename T>
__device__ __forceinline__ void block_colsum_row(const A (&acc)[V], T* __restrict__ out, int64_t k, A* sm) {
  const int lane = threadIdx.x % L, grp = threadIdx.x / L;
  constexpr int G = kBlk / L;
#pragma unroll
  for (int j = 0; j < V; ++j) sm[(grp * L + lane) * V + j] = acc[j];
  __syncthreads();
  for (int c = threadIdx.x; c < L * V && c < k; c += kBlk) {
    const int l = c / V, j = c % V;
    A s = acc_zero<A>();
    for (int g = 0; g < G; ++g) s = acc_add(s, sm[(g * L + l) * V + j]);
    if constexpr (Scalar<T>::is_complex) {
      out[c] = T{(typename Scalar<T>::real)s.x, (typename Scalar<T>::real)s.y};
    } else {
      out[c] = (T)s;
    }
  }
  __syncthreads();
}

template <typename T, int L, int V>
__global__ void __launch_bounds__(kBlk, Bps<T>::value)
cg_update_agg_kernel(int64_t nc, int64_t k, const ColState* __restrict__ cs, const T* __restrict__ dinv,
                     T* __restrict__ R, const T* __restrict__ Q,
                     const int32_t* __restrict__ agg_ptr, const int32_t* __restrict__ agg_rows,
                     T* __restrict__ rc, typename Scalar<T>::acc* __restrict__ part_rz,
                     double* __restrict__ part_rr, const int32_t* __restrict__ live) {
  if (live && *live == 0) return;  // every column converged: a no-op iteration
  typedef typename Scalar<T>::acc A;
  __shared__ A sm[kBlk * V];
  __shared__ double smr[kBlk * V];
  constexpr int G = kBlk / L;
  const int lane = threadIdx.x % L, grp = threadIdx.x / L;
  const int64_t c0 = (int64_t)lane * V;
  const bool on = c0 < k;
  alignas(16) T al[V];
  bool act[V];
#pragma unroll
  for (int j = 0; j < V; ++j) {
    act[j] = on && cs[c0 + j].active;
    al[j] = act[j] ? from_c<T>(cs[c0 + j].alpha) : s_zero(T());
  }
  alignas(16) A arz[V];
  alignas(16) double arr[V];
#pragma unroll
  for (int j = 0; j < V; ++j) { arz[j] = acc_zero<A>(); arr[j] = 0.0; }
  for (int64_t I = blockIdx.x; I < nc; I += gridDim.x) {
    alignas(16) T rs[V];
#pragma unroll
    for (int j = 0; j < V; ++j) rs[j] = s_zero(T());
    const int32_t q1 = agg_ptr[I + 1];
    int32_t q = agg_ptr[I] + grp;
    int32_t nrow = q < q1 ? agg_rows[q] : 0;
    for (; q < q1; q += G) {
      const int64_t row = nrow;
      if (q + G < q1) nrow = agg_rows[q + G];  // next row's index in flight
      if (!on) continue;
      const T d = dinv[row];
      alignas(16) T r[V], qv[V];
      ldv<T, V>(R + row * k + c0, r);
      ldv<T, V>(Q + row * k + c0, qv);
#pragma unroll
      for (int j = 0; j < V; ++j) {
        if (act[j]) r[j] = s_sub(r[j], s_mul(al[j], qv[j]));
        const T z = s_mul(d, r[j]);
        arz[j] = acc_fma(r[j], z, arz[j]);
        arr[j] += s_abs2(r[j]);
        rs[j] = s_add(rs[j], r[j]);
      }
      stv<T, V>(R + row * k + c0, r);
    }
    {
      alignas(16) A rsa[V];
#pragma unroll
      for (int j = 0; j < V; ++j) rsa[j] = to_acc(rs[j]);
      block_colsum_row<A, L, V, T>(rsa, rc + I * k, k, sm);
    }
  }
  block_colreduce<A, L, V>(arz, part_rz, k, sm);
  block_colreduce<double, L, V>(arr, part_rr, k, smr);
}

template <typename T, int L, int V>
__global__ void __launch_bounds__(kBlk, Bps<T>::value)
cg_pupdate_agg_kernel(int64_t nc, int64_t k, const ColState* __restrict__ cs, const T* __restrict__ dinv,
                      const T* __restrict__ R, T* __restrict__ P, T* __restrict__ Xs,
                      const int32_t* __restrict__ agg_ptr, const int32_t* __restrict__ agg_rows,
                      const T* __restrict__ ec) {
  constexpr int G = kBlk / L;
  const int lane = threadIdx.x % L, grp = threadIdx.x / L;
  const int64_t c0 = (int64_t)lane * V;
  if (c0 >= k) return;
  PupCols<T, V> pc;
  pc.load(cs, c0);
  if (!pc.any_act && !pc.any_upd) return;
  for (int64_t I = blockIdx.x; I < nc; I += gridDim.x) {
    alignas(16) T e[V];
    ldv<T, V>(ec + I * k + c0, e);
    const int32_t q1 = agg_ptr[I + 1];
    int32_t q = agg_ptr[I] + grp;
    int32_t nrow = q < q1 ? agg_rows[q] : 0;
    for (; q < q1; q += G) {
      const int64_t row = nrow;
      if (q + G < q1) nrow = agg_rows[q + G];
      pc.row(Xs + row * k + c0, P + row * k + c0, R + row * k + c0, dinv[row], e);
    }
  }
}

// ----------------------------------------------------------- finalizers
__device__ __forceinline__ cdouble cdiv(cdouble a, cdouble b) {
  const double d = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
__device__ __forceinline__ bool finite_c(cdouble a) { return isfinite(a.x) && isfinite(a.y); }

// One warp per column: lanes stride over the per-block partials (4 loads in
// flight per lane), then a fixed shuffle tree; deterministic for a fixed grid.
__device__ __forceinline__ double wsum(double v) { return warp_sum(v); }
__device__ __forceinline__ cdouble wsum(cdouble v) { return make_double2(warp_sum(v.x), warp_sum(v.y)); }

template <typename A>
__device__ __forceinline__ cdouble sum_part(const A* __restrict__ part, int nb, int64_t k, int64_t c, int lane) {
  A s0 = acc_zero<A>(), s1 = acc_zero<A>(), s2 = acc_zero<A>(), s3 = acc_zero<A>();
  int b = lane;
  for (; b + 96 < nb; b += 128) {
    s0 = acc_add(s0, part[(int64_t)b * k + c]);
    s1 = acc_add(s1, part[(int64_t)(b + 32) * k + c]);
    s2 = acc_add(s2, part[(int64_t)(b + 64) * k + c]);
    s3 = acc_add(s3, part[(int64_t)(b + 96) * k + c]);
  }
  for (; b < nb; b += 32) s0 = acc_add(s0, part[(int64_t)b * k + c]);
  return to_c(wsum(acc_add(acc_add(s0, s1), acc_add(s2, s3))));
}

#define RB_FIN_WARP()                                   \
  const int lane = threadIdx.x & 31;                    \
  const int64_t c = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); \
  if (c >= k) return;

// after init: rz, rr0; a column is active iff its rhs is nonzero and enabled
template <typename A>
__global__ void fin_init_kernel(int64_t k, int nb, const A* part_rz, const double* part_rr, ColState* cs,
                                const int32_t* __restrict__ enable, const OuterState* __restrict__ os,
                                int32_t* __restrict__ live) {
  RB_FIN_WARP();
  const cdouble rz = sum_part<A>(part_rz, nb, k, c, lane);
  const double rr = sum_part<double>(part_rr, nb, k, c, lane).x;
  if (lane) return;
  ColState s = cs[c];
  s.rz = rz;
  s.rr = rr;
  s.rr0 = s.rr;
  s.active = (enable == nullptr || enable[c]) && s.rr > 0.0;
  s.status = 0;
  s.iters = 0;
  s.tol2 = os ? os[c].itol2 : -1.0;
  s.alpha = make_double2(0, 0);
  s.beta = make_double2(0, 0);
  s.upd = 0;
  cs[c] = s;
  if (s.active) atomicAdd(live, 1);
}

// The per-iteration finalizers take one block of kFinThreads per column: each
// thread sums the partials b = tid, tid + kFinThreads, ... (two accumulators),
// then warps and the block's warps are added in fixed order (deterministic),
// 8 times shorter load chains than one warp per column (the update kernel
// leaves 1184 partials per column).  The sum is valid in thread 0.
constexpr int kFinThreads = 256;
template <typename A>
__device__ __forceinline__ cdouble block_sum_part(const A* __restrict__ part, int nb, int64_t k, int64_t c) {
  __shared__ cdouble red[kFinThreads / 32];
  A s0 = acc_zero<A>(), s1 = acc_zero<A>();
  int b = threadIdx.x;
  for (; b + kFinThreads < nb; b += 2 * kFinThreads) {
    s0 = acc_add(s0, part[(int64_t)b * k + c]);
    s1 = acc_add(s1, part[(int64_t)(b + kFinThreads) * k + c]);
  }
  for (; b < nb; b += kFinThreads) s0 = acc_add(s0, part[(int64_t)b * k + c]);
  const cdouble w = to_c(wsum(acc_add(s0, s1)));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = w;
  __syncthreads();
  cdouble t = make_double2(0.0, 0.0);
  if (threadIdx.x == 0)
    for (int q = 0; q < kFinThreads / 32; ++q) t = make_double2(t.x + red[q].x, t.y + red[q].y);
  __syncthreads();  // red is reused by the next sum
  return t;
}

// also clears the live-column slot that this iteration's fin_beta counts
// into (its previous readers, the kernels of the iteration before, are done)
template <typename A>
__global__ void __launch_bounds__(kFinThreads) fin_alpha_kernel(int64_t k, int nb, const A* part_pq, ColState* cs,
                                                               int32_t* __restrict__ clear) {
  if (clear && blockIdx.x == 0 && threadIdx.x == 0) *clear = 0;
  const int64_t c = blockIdx.x;
  if (c >= k) return;
  if (!cs[c].active) {  // uniform over the block; no x update in this iteration's p-update
    if (threadIdx.x == 0) cs[c].upd = 0;
    return;
  }
  const cdouble pq = block_sum_part<A>(part_pq, nb, k, c);
  if (threadIdx.x) return;
  ColState s = cs[c];
  s.pq = pq;
  if (!finite_c(s.pq) || (s.pq.x == 0.0 && s.pq.y == 0.0)) {
    s.active = 0;
    s.status = 2;
    s.alpha = make_double2(0, 0);
    s.upd = 0;
  } else {
    s.alpha = cdiv(s.rz, s.pq);
    s.upd = 1;
  }
  cs[c] = s;
}

// beta = rz_new / rz; convergence ||r|| <= tol ||r0||; counts active columns.
// With a coarse space rz_new adds the coarse part (P^T r).(X P^T r), whose
// per-block partials are part_c (nbc blocks).
template <typename A>
__global__ void __launch_bounds__(kFinThreads) fin_beta_kernel(int64_t k, int nb, const A* part_rz,
                                                              const double* part_rr, ColState* cs, double tol2,
                                                              int32_t* nactive, const A* part_c, int nbc) {
  const int64_t c = blockIdx.x;
  if (c >= k || !cs[c].active) return;  // uniform over the block
  cdouble rzn = block_sum_part<A>(part_rz, nb, k, c);
  if (part_c) {
    const cdouble rc = block_sum_part<A>(part_c, nbc, k, c);
    rzn = make_double2(rzn.x + rc.x, rzn.y + rc.y);
  }
  const double rr = block_sum_part<double>(part_rr, nb, k, c).x;
  if (threadIdx.x) return;
  ColState s = cs[c];
  s.iters += 1;
  s.rr = rr;
  if (!finite_c(rzn) || !isfinite(rr)) {
    s.active = 0;
    s.status = 2;
  } else if (rr <= (s.tol2 >= 0.0 ? s.tol2 : tol2) * s.rr0) {
    s.active = 0;
  } else if (s.rz.x == 0.0 && s.rz.y == 0.0) {
    s.active = 0;
    s.status = 2;
  } else {
    s.beta = cdiv(rzn, s.rz);
    s.rz = rzn;
  }
  cs[c] = s;
  if (s.active) atomicAdd(nactive, 1);
}

// --------------------------------------------------- refinement kernels

// refinement state before the first sweep from ||b||^2: a zero column is
// done (exactly zero solution); a non-finite one is done with the
// non-finite outcome (3), never counted as converged
__device__ __forceinline__ OuterState outer_start(double s) {
  OuterState o;
  const bool fin = isfinite(s);
  o.bnorm = sqrt(s);
  // no previous sweep yet: the first residual can never count as stagnation
  o.relres = !fin ? s : (s > 0.0) ? 1e300 : 0.0;
  o.prev = 1e300;
  o.scale = 0.0;
  o.itol2 = -1.0;
  o.active = fin && s > 0.0;
  o.done = !fin ? 3 : (s > 0.0) ? 0 : 1;
  return o;
}

__global__ void fin_bnorm_kernel(int64_t k, int nb, const double* part, OuterState* os) {
  RB_FIN_WARP();
  const double s = sum_part<double>(part, nb, k, c, lane).x;
  if (lane) return;
  os[c] = outer_start(s);
}

// A sweep normally solves its correction to inner_tol.  The sweep that will
// bring a column to the target solves to 1e-2 * tol / relres instead (not
// below itol_min, the inner precision's reach): it over-solves past the FP64
// floor, so that small far-field entries of the solution, which a global
// residual norm barely sees, converge as well.
__global__ void fin_outer_kernel(int64_t k, int nb, const double* part, OuterState* os, double tol,
                                 double stall, double inner_tol, double itol_min, int32_t* nactive) {
  RB_FIN_WARP();
  if (!os[c].active) return;
  const double s = sum_part<double>(part, nb, k, c, lane).x;
  if (lane) return;
  OuterState o = os[c];
  const double rel = sqrt(s) / o.bnorm;
  o.prev = o.relres;
  o.relres = rel;
  if (!isfinite(rel)) {  // NaN/Inf in the matrix, the data or a correction
    o.active = 0;
    o.done = 3;
  } else if (!(rel > tol)) {
    o.active = 0;
    o.done = 1;
  } else if (rel > stall * o.prev) {
    o.active = 0;
    o.done = 2;
  } else {
    o.scale = 1.0 / sqrt(s);
    double it = inner_tol;
    if (rel * inner_tol < 10.0 * tol) it = fmax(fmin(inner_tol, 1e-2 * tol / rel), itol_min);
    o.itol2 = it * it;
  }
  os[c] = o;
  if (o.active) atomicAdd(nactive, 1);
}

// The state that scales row `i`'s entry of column c: the column's own, or
// with stacked instances (rinst given) that of the row's (instance, column)
__device__ __forceinline__ const OuterState& row_state(const OuterState* os, const int32_t* __restrict__ rinst,
                                                       int64_t i, int64_t k, int64_t c) {
  return rinst ? os[(int64_t)rinst[i / k] * k + c] : os[c];
}

// r_inner = T(R64 * scale) for active columns, 0 elsewhere
template <typename T64, typename T>
__global__ void cast_scale_kernel(int64_t n, int64_t k, const T64* __restrict__ R64, const OuterState* os,
                                  const int32_t* __restrict__ rinst, T* __restrict__ R) {
  const int64_t total = n * k;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = i % k;
    const OuterState& o = row_state(os, rinst, i, k, c);
    const double s = o.active ? o.scale : 0.0;
    T64 v = R64[i];
    if constexpr (Scalar<T>::is_complex) {
      R[i] = T{(typename Scalar<T>::real)(v.x * s), (typename Scalar<T>::real)(v.y * s)};
    } else {
      R[i] = (T)(v * s);
    }
  }
}

// X64 += D / scale for active columns
template <typename T64, typename T>
__global__ void correct_kernel(int64_t n, int64_t k, const T* __restrict__ D, const OuterState* os,
                               const int32_t* __restrict__ rinst, T64* __restrict__ X) {
  const int64_t total = n * k;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = i % k;
    const OuterState& o = row_state(os, rinst, i, k, c);
    if (!o.active) continue;
    const double inv = 1.0 / o.scale;
    T d = D[i];
    if constexpr (Scalar<T>::is_complex) {
      X[i].x += (double)d.x * inv;
      X[i].y += (double)d.y * inv;
    } else {
      X[i] += (double)d * inv;
    }
  }
}

constexpr int64_t kMaxCols = 128;  // columns per Krylov block

// ------------------------------------------- stacked independent instances
// With a batch of independent systems stacked block-diagonally, the
// refinement keeps one OuterState per (instance, column): each instance is
// tested against its own ||b_i||, its correction right-hand side is scaled
// to unit norm on its own rows, and it stops being corrected once its
// columns are done, whatever the other instances do.  The inner Krylov
// sweep still runs on whole columns; its per-column state is the summary
// of the column's instances (active if any is, the tightest inner tolerance).

__device__ __forceinline__ double sq_abs(double v) { return v * v; }
__device__ __forceinline__ double sq_abs(cdouble v) { return v.x * v.x + v.y * v.y; }

// out[i * k + c] = sum over instance i's rows of |X[r][c]|^2: one block per
// instance, warps over rows, lanes over columns, summed in a fixed order
constexpr int kSegWarps = 8;
template <typename T64>
__global__ void __launch_bounds__(kSegWarps * 32)
seg_norm_kernel(int64_t ninst, int64_t k, const int64_t* __restrict__ row_ptr, const T64* __restrict__ X,
                double* __restrict__ out) {
  __shared__ double sm[kSegWarps][kMaxCols];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int64_t i = blockIdx.x; i < ninst; i += gridDim.x) {
    double a[kMaxCols / 32];
#pragma unroll
    for (int q = 0; q < kMaxCols / 32; ++q) a[q] = 0.0;
    const int64_t r1 = row_ptr[i + 1];
    for (int64_t r = row_ptr[i] + w; r < r1; r += kSegWarps) {
      const T64* xr = X + r * k;
#pragma unroll
      for (int q = 0; q < kMaxCols / 32; ++q)
        if (lane + 32 * q < k) a[q] += sq_abs(xr[lane + 32 * q]);
    }
#pragma unroll
    for (int q = 0; q < kMaxCols / 32; ++q)
      if (lane + 32 * q < k) sm[w][lane + 32 * q] = a[q];
    __syncthreads();
    for (int64_t c = threadIdx.x; c < k; c += blockDim.x) {
      double t = 0.0;
#pragma unroll
      for (int q = 0; q < kSegWarps; ++q) t += sm[q][c];
      out[i * k + c] = t;
    }
    __syncthreads();
  }
}

__global__ void seg_bnorm_kernel(int64_t m, const double* __restrict__ s2, OuterState* __restrict__ seg) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= m) return;
  seg[j] = outer_start(s2[j]);
}

// the rules of fin_outer_kernel, per (instance, column)
__global__ void seg_outer_kernel(int64_t m, const double* __restrict__ s2, OuterState* __restrict__ seg, double tol,
                                 double stall, double inner_tol, double itol_min) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= m || !seg[j].active) return;
  const double s = s2[j];
  OuterState o = seg[j];
  const double rel = sqrt(s) / o.bnorm;
  o.prev = o.relres;
  o.relres = rel;
  if (!isfinite(rel)) {
    o.active = 0;
    o.done = 3;
  } else if (!(rel > tol)) {
    o.active = 0;
    o.done = 1;
  } else if (rel > stall * o.prev) {
    o.active = 0;
    o.done = 2;
  } else {
    o.scale = 1.0 / sqrt(s);
    double it = inner_tol;
    if (rel * inner_tol < 10.0 * tol) it = fmax(fmin(inner_tol, 1e-2 * tol / rel), itol_min);
    o.itol2 = it * it;
  }
  seg[j] = o;
}

// column summary of the instances' states; counts the active columns
__global__ void seg_summary_kernel(int64_t ninst, int64_t k, const OuterState* __restrict__ seg,
                                   OuterState* __restrict__ os, int32_t* __restrict__ nactive) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= k) return;
  OuterState o;
  o.bnorm = 0.0;
  o.relres = 0.0;
  o.prev = 0.0;
  o.scale = 1.0;
  o.itol2 = -1.0;
  o.active = 0;
  bool nonfinite = false, open = false, stalled = false;
  for (int64_t i = 0; i < ninst; ++i) {
    const OuterState& q = seg[i * k + c];
    if (isfinite(q.relres)) o.relres = fmax(o.relres, q.relres);
    else nonfinite = true;
    nonfinite |= q.done == 3;
    open |= q.done == 0;
    stalled |= q.done == 2;
    if (q.active) {
      o.itol2 = o.active ? fmin(o.itol2, q.itol2) : q.itol2;
      o.active = 1;
    }
  }
  // the column's worst instance: non-finite, still open, stalled, converged
  o.done = nonfinite ? 3 : open ? 0 : stalled ? 2 : 1;
  if (nonfinite) o.relres = __longlong_as_double(0x7ff0000000000000LL);  // +inf
  os[c] = o;
  if (o.active) atomicAdd(nactive, 1);
}

// per-instance outcome: 0 converged, 1 not converged within the caps,
// 2 Krylov breakdown, 3 non-finite residual; relres per (instance, column)
__global__ void seg_status_kernel(int64_t ninst, int64_t k, int64_t ncol, const OuterState* __restrict__ seg,
                                  const ColState* __restrict__ cs, const int32_t* __restrict__ counter,
                                  int32_t* __restrict__ status, double* __restrict__ relres) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= ninst) return;
  // 4: a bounded in-kernel wait of the SpMM gave up (results not valid)
  int32_t st = counter[2] ? 4 : 0;
  for (int64_t c = 0; c < ncol; ++c) {
    const OuterState& q = seg[i * k + c];
    if (relres) relres[i * ncol + c] = q.relres;
    int32_t v = 0;
    if (q.done == 3) v = 3;
    else if (cs[c].status == 2 && q.relres > 1e-10 && q.done != 1) v = 2;
    else if (q.done == 0 || (q.done == 2 && q.relres > 1e-10)) v = 1;
    st = max(st, v);
  }
  status[i] = st;
}

// squared column norms of a real FP64 n x k array
template <int L, int V>
__global__ void __launch_bounds__(kBlk, 4)
colnorm_kernel(int64_t n, int64_t k, const double* __restrict__ B, double* __restrict__ part) {
  __shared__ double sm[kBlk * V];
  const int lane = threadIdx.x % L;
  const int64_t c0 = (int64_t)lane * V;
  const bool on = c0 < k;
  const int64_t groups = (int64_t)gridDim.x * (kBlk / L);
  alignas(16) double acc[V];
#pragma unroll
  for (int j = 0; j < V; ++j) acc[j] = 0.0;
  for (int64_t row = blockIdx.x * (int64_t)(kBlk / L) + threadIdx.x / L; row < n; row += groups) {
    if (!on) continue;
#pragma unroll
    for (int j = 0; j < V; ++j) {
      const double b = B[row * k + c0 + j];
      acc[j] += b * b;
    }
  }
  block_colreduce<double, L, V>(acc, part, k, sm);
}

// ------------------------------------------------------------- dispatch
struct Shape {
  int L, V;
  unsigned grid;
  int S = 1;  // column slices of the SpMM (see spmm_kernel)
};

static int64_t num_sms() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    if (sms * 5 > kGridMax) sms = kGridMax / 5;  // partials arrays hold kGridMax blocks
  }
  return sms;
}

static Shape pick_shape(int64_t n, int64_t k, int bps) {
  Shape s;
  s.V = (k % 4 == 0) ? 4 : (k % 2 == 0) ? 2 : 1;
  int need = (int)ceil_div(k, s.V);
  s.L = need <= 4 ? 4 : need <= 8 ? 8 : need <= 16 ? 16 : 32;
  // one resident wave: every block stays on its SM for the whole kernel
  s.grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(num_sms() * bps, ceil_div(n, kBlk / s.L)));
  return s;
}

// Column counts the lane layout of pick_shape covers (L V >= k): up to 32
// columns of any count, even counts up to 64, multiples of 4 up to 128.  A
// solve of another count runs on a copy padded with zero columns to the next
// multiple of 4 (zero right-hand sides stay inactive and exactly zero).
static int64_t solve_cols(int64_t k) {
  if (k <= 32 || k % 4 == 0 || (k % 2 == 0 && k <= 64)) return k;
  return ceil_div(k, 4) * 4;
}
static bool shape_covers(const Shape& s, int64_t k) { return (int64_t)s.S * s.L * s.V >= k; }
}  // namespace rb
#include "rb_spmm_blk.cuh"
namespace rb {

// D[i][c] = S[i][c] for c < ks, 0 beyond (row-major, ld ks and kd)
template <typename T>
__global__ void copy_cols_kernel(int64_t n, int64_t ks, int64_t kd, const T* __restrict__ S, T* __restrict__ D) {
  const int64_t total = n * kd;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / kd, c = i % kd;
    D[i] = c < ks ? S[r * ks + c] : s_zero(T());
  }
}

// Y = A X for any column count: a warp per row, lanes over columns (plain
// loads; rb_spmm's path for counts the vectorised layout does not cover)
template <typename T>
__global__ void spmm_any_kernel(int64_t n, int64_t k, const int32_t* __restrict__ indptr,
                                const int32_t* __restrict__ indices, const T* __restrict__ val,
                                const T* __restrict__ X, T* __restrict__ Y) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t row = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); row < n; row += warps) {
    const int32_t b = indptr[row], e = indptr[row + 1];
    for (int64_t c = lane; c < k; c += 32) {
      T y = s_zero(T());
      for (int32_t p = b; p < e; ++p) y = s_fma(val[p], X[(int64_t)indices[p] * k + c], y);
      Y[row * k + c] = y;
    }
  }
}

// SpMM shape: complex64 at 128 columns takes two 64-column slices (2 values
// of 8 bytes per lane, 8 gathers in flight), measured 23% faster per launch
// than one slice of 4 values with 4 gathers in flight
template <typename T>
static Shape pick_spmm_shape(int64_t n, int64_t k) {
  if (std::is_same<T, cfloat>::value && k == 128) {
    Shape s;
    s.L = 32;
    s.V = 2;
    s.S = 2;
    s.grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(num_sms() * BpsSpmm<T>::value,
                                                               ceil_div(2 * n, kBlk / s.L)));
    return s;
  }
  return pick_shape(n, k, BpsSpmm<T>::value);
}

#define RB_DISPATCH_LV(sh, FN)                       \
  switch (sh.L * 8 + sh.V) {                         \
    case 4 * 8 + 1: FN(4, 1); break;                 \
    case 4 * 8 + 2: FN(4, 2); break;                 \
    case 4 * 8 + 4: FN(4, 4); break;                 \
    case 8 * 8 + 1: FN(8, 1); break;                 \
    case 8 * 8 + 2: FN(8, 2); break;                 \
    case 8 * 8 + 4: FN(8, 4); break;                 \
    case 16 * 8 + 1: FN(16, 1); break;               \
    case 16 * 8 + 2: FN(16, 2); break;               \
    case 16 * 8 + 4: FN(16, 4); break;               \
    case 32 * 8 + 1: FN(32, 1); break;               \
    case 32 * 8 + 2: FN(32, 2); break;               \
    case 32 * 8 + 4: FN(32, 4); break;               \
    default: return fail(RB_EARG, "bad shape");      \
  }

// live: the live-column count the iteration kernels read (NULL outside the
// Krylov loop)
template <typename T, int EPI>
int spmm_t(const rb_csr& A, const T* val, const T* X, T* Y, const double* B, void* part, int64_t k,
           const Shape& sh, cudaStream_t st, const int32_t* live = nullptr) {
  const bool o32 = (uint64_t)A.n * (uint64_t)k < (1ull << 31);
  if (sh.S == 2) {
    if (sh.L != 32 || sh.V != 2 || k != 128) return fail(RB_EARG, "bad sliced SpMM shape");
    if (o32)
      spmm_kernel<T, 32, 2, EPI, 2, true><<<sh.grid, kBlk, 0, st>>>(A.n, k, A.indptr, A.indices, val, X, Y, B, part, live);
    else
      spmm_kernel<T, 32, 2, EPI, 2, false><<<sh.grid, kBlk, 0, st>>>(A.n, k, A.indptr, A.indices, val, X, Y, B, part, live);
    RB_LAUNCH_CHECK();
    return RB_OK;
  }
  if (sh.L == 32 && !o32) {  // offsets beyond int32: the 64-bit index arithmetic
#define RB_SPMM(L_, V_) \
  spmm_kernel<T, L_, V_, EPI, 1, false><<<sh.grid, kBlk, 0, st>>>(A.n, k, A.indptr, A.indices, val, X, Y, B, part, live)
    RB_DISPATCH_LV(sh, RB_SPMM);
#undef RB_SPMM
    RB_LAUNCH_CHECK();
    return RB_OK;
  }
#define RB_SPMM(L_, V_) \
  spmm_kernel<T, L_, V_, EPI><<<sh.grid, kBlk, 0, st>>>(A.n, k, A.indptr, A.indices, val, X, Y, B, part, live)
  RB_DISPATCH_LV(sh, RB_SPMM);
#undef RB_SPMM
  RB_LAUNCH_CHECK();
  return RB_OK;
}

// Row-group SpMM launch (k = 32 V columns); grid = resident blocks on all SMs
static bool grp_cols_ok(int64_t k) { return k == 32 || k == 64 || k == 128; }

template <typename T, int V, int EPI>
static int spmm_grp_v(const rb_csr& A, const T* val, const GroupPlan& gp, const T* X, T* Y, const double* B,
                      void* part, int32_t* err, unsigned* grid_out, cudaStream_t st, const int32_t* live) {
  static int bps = 0;  // resident blocks per SM of this instantiation
  constexpr size_t smem = grp_smem_bytes<T>();
  if (!bps) {
    RB_CUDA_TRY(cudaFuncSetAttribute(spmm_grp_kernel<T, V, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
    int nb = 0;
    RB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, spmm_grp_kernel<T, V, EPI>, kGrpWarps * 32,
                                                              smem));
    bps = std::max(1, nb);
  }
  const int64_t grid = std::max<int64_t>(
      1, std::min<int64_t>(std::min<int64_t>(num_sms() * bps, ceil_div(gp.ng, kGrpWarps)), kGridMax));
  spmm_grp_kernel<T, V, EPI><<<(unsigned)grid, kGrpWarps * 32, smem, st>>>(A.n, A.indptr, val, gp, X, Y, B, part,
                                                                            err, live);
  RB_LAUNCH_CHECK();
  *grid_out = (unsigned)grid;
  return RB_OK;
}

template <typename T, int EPI>
static int spmm_grp(const rb_csr& A, const T* val, const GroupPlan& gp, const T* X, T* Y, const double* B,
                    void* part, int64_t k, int32_t* err, unsigned* grid_out, cudaStream_t st,
                    const int32_t* live) {
  switch (k) {
    case 32: return spmm_grp_v<T, 1, EPI>(A, val, gp, X, Y, B, part, err, grid_out, st, live);
    case 64: return spmm_grp_v<T, 2, EPI>(A, val, gp, X, Y, B, part, err, grid_out, st, live);
    case 128: return spmm_grp_v<T, 4, EPI>(A, val, gp, X, Y, B, part, err, grid_out, st, live);
    default: return fail(RB_EARG, "row-group SpMM: %lld columns", (long long)k);
  }
}

template <typename T, int EPI>
static int spmm_pair(const rb_csr& A, const T* val, const GroupPlan& gp, const T* X, T* Y, void* part,
                     int64_t k, unsigned* grid_out, cudaStream_t st, const int32_t* live) {
  if (!pair_cols_ok<T>(k) || A.n * k >= (int64_t(1) << 31))
    return fail(RB_EARG, "row-pair SpMM: %lld columns", (long long)k);
  const unsigned grid = (unsigned)std::max<int64_t>(
      1, std::min<int64_t>(num_sms() * BpsSpmm<T>::value, ceil_div(gp.ng * PairCfg<T>::S, kBlk / 32)));
  spmm_pair_kernel<T, EPI><<<grid, kBlk, 0, st>>>(A.n, k, A.indptr, val, gp, X, Y, part, live);
  RB_LAUNCH_CHECK();
  *grid_out = grid;
  return RB_OK;
}

// union lists of the row groups: count, scan, fill
template <int G>
static int build_group_plan(const rb_csr& A, int32_t* gcnt, int32_t* gptr, int32_t* ucol, uint8_t* umask,
                            void* scan_work, size_t scan_bytes, GroupPlan* gp, cudaStream_t st) {
  const int64_t ng = ceil_div(A.n, G);
  const unsigned grid = (unsigned)std::min<int64_t>(ceil_div(ng, 128), 148 * 32);
  group_union_kernel<G, false><<<grid, 128, 0, st>>>(A.n, A.indptr, A.indices, gcnt, nullptr, nullptr);
  RB_LAUNCH_CHECK();
  RB_TRY(scan_exclusive(gcnt, gptr, ng, scan_work, scan_bytes, st));
  group_union_kernel<G, true><<<grid, 128, 0, st>>>(A.n, A.indptr, A.indices, gptr, ucol, umask);
  RB_LAUNCH_CHECK();
  *gp = GroupPlan{gptr, ucol, umask, ng};
  return RB_OK;
}

// Workspace carving --------------------------------------------------------
struct Carver {
  char* p;
  size_t left;
  size_t used = 0;
  template <typename X> X* take(size_t count) {
    size_t bytes = (count * sizeof(X) + 255) / 256 * 256;
    used += bytes;
    if (bytes > left) return nullptr;
    X* r = reinterpret_cast<X*>(p);
    p += bytes;
    left -= bytes;
    return r;
  }
};

template <typename T64, typename T>
struct SolveBufs {
  T64* R64;
  T *Xs, *R, *P, *Q;
  void* part_a;   // kGridMax x k acc
  double* part_b; // kGridMax x k double
  ColState* cs;
  OuterState* os;
  int32_t* enable;
  int32_t* counter;  // [1] active outer columns, [2] SpMM wait timeout, [4..5] live inner columns
                     // (two slots, alternating per iteration), [6..7] their values at burst ends
  // row-group plan of the SpMM (k = 32, 64 or 128 columns)
  int32_t *gcnt, *gptr, *ucol;
  uint8_t* umask;
  void* scan_work;
  size_t scan_bytes;
};

// per-(instance, column) refinement state of a stacked batch
struct SegBufs {
  const rb_instances* in = nullptr;
  int64_t ncol = 0;        // the caller's columns (relres layout)
  double* s2 = nullptr;    // ninst x k squared norms
  OuterState* seg = nullptr;  // ninst x k
};
static size_t seg_carve(Carver& cv, SegBufs& sb, int64_t ninst, int64_t k) {
  sb.s2 = cv.take<double>(ninst * k);
  sb.seg = cv.take<OuterState>(ninst * k);
  return cv.used;
}

template <typename T64, typename T>
static size_t carve(Carver& cv, SolveBufs<T64, T>& b, int64_t n, int64_t nnz, int64_t k) {
  b.R64 = cv.take<T64>(n * k);
  b.Xs = cv.take<T>(n * k);
  b.R = cv.take<T>(n * k);
  b.P = cv.take<T>(n * k);
  b.Q = cv.take<T>(n * k);
  b.part_a = cv.take<cdouble>((size_t)kGridMax * k);
  b.part_b = cv.take<double>((size_t)kGridMax * k);
  b.cs = cv.take<ColState>(k);
  b.os = cv.take<OuterState>(k);
  b.enable = cv.take<int32_t>(k);
  b.counter = cv.take<int32_t>(8);
  const int64_t ng = ceil_div(n, GrpCfg<T>::G);
  b.gcnt = cv.take<int32_t>(ng + 1);
  b.gptr = cv.take<int32_t>(ng + 1);
  b.ucol = cv.take<int32_t>(std::max<int64_t>(nnz, 1));
  b.umask = cv.take<uint8_t>(std::max<int64_t>(nnz, 1));
  b.scan_bytes = scan_work_bytes(ng);
  b.scan_work = cv.take<char>(b.scan_bytes);
  return cv.used;
}

// Inner Jacobi-PCG / COCG on A x = R (scaled residuals), x -> b.Xs.
// Optional per-kernel timing of the Krylov loop with CUDA events on the
// launching stream (SpMM and vector-update kernels), read at the host sync
// points the loop already has.
struct KernelTimer {
  bool on = false;
  std::vector<cudaEvent_t> ev;
  int used = 0;
  double spmm_ms = 0, upd_ms = 0, coarse_ms = 0;
  int spmm_n = 0, upd_n = 0, coarse_n = 0;
  bool with_coarse = false;
  int ensure(int n) {
    while ((int)ev.size() < n) {
      cudaEvent_t e;
      RB_CUDA_TRY(cudaEventCreate(&e));
      ev.push_back(e);
    }
    return RB_OK;
  }
  int record(cudaStream_t st) {
    if (!on) return RB_OK;
    RB_TRY(ensure(used + 1));
    RB_CUDA_TRY(cudaEventRecord(ev[used++], st));
    return RB_OK;
  }
  // events come in fours: before spmm, after spmm, after update, after the
  // coarse correction (restriction, coarse product, dot)
  int harvest() {
    if (!on) return RB_OK;
    for (int i = 0; i + 3 < used; i += 4) {
      float a = 0, b = 0, c = 0;
      RB_CUDA_TRY(cudaEventElapsedTime(&a, ev[i], ev[i + 1]));
      RB_CUDA_TRY(cudaEventElapsedTime(&b, ev[i + 1], ev[i + 2]));
      RB_CUDA_TRY(cudaEventElapsedTime(&c, ev[i + 2], ev[i + 3]));
      spmm_ms += a;
      upd_ms += b;
      spmm_n++;
      upd_n++;
      if (with_coarse) {
        coarse_ms += c;
        coarse_n++;
      }
    }
    used = 0;
    return RB_OK;
  }
  ~KernelTimer() {
    for (auto e : ev) cudaEventDestroy(e);
  }
};

// Host side of the burst pipeline: one event per snapshot slot and a side
// stream (per device, created once) on which the 4-byte snapshot is read
// back, so that the read waits for its own burst only, not for the burst
// queued behind it on the solve's stream.
static cudaStream_t side_stream() {
  static cudaStream_t streams[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  if (!streams[dev]) cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking);
  return streams[dev];
}

struct BurstSync {
  cudaEvent_t ev[2] = {nullptr, nullptr};
  cudaStream_t side = nullptr;
  int init() {
    side = side_stream();
    if (!side) return fail(RB_ECUDA, "rb_femsolve: no side stream");
    for (auto& e : ev) RB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return RB_OK;
  }
  // the live count at the end of the burst recorded in slot s
  int read(int s, const int32_t* snap, int32_t* v) {
    RB_CUDA_TRY(cudaEventSynchronize(ev[s]));
    RB_CUDA_TRY(cudaMemcpyAsync(v, snap + s, sizeof(int32_t), cudaMemcpyDeviceToHost, side));
    RB_CUDA_TRY(cudaStreamSynchronize(side));
    return RB_OK;
  }
  ~BurstSync() {
    for (auto e : ev)
      if (e) cudaEventDestroy(e);
  }
};

template <typename T>
static int inner_solve(const rb_csr& A, const T* val, const T* dinv, int64_t k, const Shape& sh, const Shape& shs,
                       void* part_a,
                       double* part_b, T* Xs, T* R, T* P, T* Q, ColState* cs, const int32_t* enable,
                       const OuterState* os, int32_t* counter, double tol, int maxiter, int check_every,
                       int* iters_out,
                       int* launches, KernelTimer& tm, const GroupPlan* gp, const RowGroupsDev* rg,
                       const CoarseOp<T>* co, cudaStream_t st) {
  typedef typename Scalar<T>::acc Acc;
  const int64_t n = A.n;
  const unsigned fg = (unsigned)ceil_div(k, 8);
  const int32_t* agg = co ? co->agg : nullptr;
  const T* ec = co ? co->ec : nullptr;
  const Acc* part_c = co ? (const Acc*)co->part : nullptr;
  // blocks of the aggregate-ordered kernels: two waves of resident blocks
  // (the second evens out aggregates of unequal size), within the partials
  const unsigned agrid = co ? (unsigned)std::max<int64_t>(1, std::min<int64_t>(co->nc, std::min<int64_t>(
                                                                   2 * (int64_t)sh.grid, kGridMax)))
                            : 0u;
  const unsigned ugrid = (co && AggOrder<T>::value) ? agrid : sh.grid;  // blocks of the update kernel (partials)
  if (co) {
    RB_TRY(coarse_apply<T>(*co, R, k, st));
    *launches += 3;
  }
  // live-column count: iteration i's kernels read slot rd and return at once
  // when it is 0; its fin_beta counts the columns still active into the
  // other slot (cleared by its fin_alpha), which the next iteration reads
  int32_t* slot[2] = {counter + 4, counter + 5};
  int32_t* snap = counter + 6;
  int rd = 1;
  RB_CUDA_TRY(cudaMemsetAsync(slot[rd], 0, sizeof(int32_t), st));
#define RB_INIT(L_, V_) \
  cg_init_kernel<T, L_, V_><<<sh.grid, kBlk, 0, st>>>(n, k, dinv, R, P, Xs, (Acc*)part_a, part_b, agg, ec)
  RB_DISPATCH_LV(sh, RB_INIT);
#undef RB_INIT
  RB_LAUNCH_CHECK();
  fin_init_kernel<Acc><<<fg, 256, 0, st>>>(k, (int)sh.grid, (const Acc*)part_a, part_b, cs, enable, os, slot[rd]);
  RB_LAUNCH_CHECK();
  *launches += 2;
  const double tol2 = tol * tol;
  auto enqueue_burst = [&](int burst) -> int {
    for (int b = 0; b < burst; ++b) {
      const int32_t* live = slot[rd];
      int32_t* next = slot[rd ^ 1];
      RB_TRY(tm.record(st));
      unsigned nb = shs.grid;
      if (rg) {
        if constexpr (BlkOn<T>::value) {
          RB_TRY((spmm_blk<T>(*rg, P, Q, part_a, k, &nb, st, live)));
        } else {
          return fail(RB_EARG, "blocked SpMM: unsupported scalar type");
        }
      } else if (gp) {
        if constexpr (PairCfg<T>::enabled) {
          RB_TRY((spmm_pair<T, EPI_PQDOT>(A, val, *gp, P, Q, part_a, k, &nb, st, live)));
        } else {
          RB_TRY((spmm_grp<T, EPI_PQDOT>(A, val, *gp, P, Q, nullptr, part_a, k, counter + 2, &nb, st, live)));
        }
      } else {
        RB_TRY((spmm_t<T, EPI_PQDOT>(A, val, P, Q, nullptr, part_a, k, shs, st, live)));
      }
      RB_TRY(tm.record(st));
      fin_alpha_kernel<Acc><<<(unsigned)k, kFinThreads, 0, st>>>(k, (int)nb, (const Acc*)part_a, cs, next);
      if (co && AggOrder<T>::value) {
        // aggregate order: the update also restricts the new r to rc
#define RB_UPD(L_, V_)                                                                                           \
  cg_update_agg_kernel<T, L_, V_><<<agrid, kBlk, 0, st>>>(co->nc, k, cs, dinv, R, Q, co->agg_ptr, co->agg_rows, \
                                                         co->rc, (Acc*)part_a, part_b, live)
        RB_DISPATCH_LV(sh, RB_UPD);
#undef RB_UPD
      } else {
#define RB_UPD(L_, V_)                                                                                           \
  cg_update_kernel<T, L_, V_><<<sh.grid, kBlk, 0, st>>>(n, k, cs, dinv, R, Q, (Acc*)part_a, part_b, live)
        RB_DISPATCH_LV(sh, RB_UPD);
#undef RB_UPD
      }
      RB_TRY(tm.record(st));
      if (co) {
        RB_TRY(coarse_apply<T>(*co, AggOrder<T>::value ? nullptr : R, k, st, live));
        *launches += AggOrder<T>::value ? 2 : 3;
      }
      RB_TRY(tm.record(st));
      fin_beta_kernel<Acc><<<(unsigned)k, kFinThreads, 0, st>>>(k, (int)ugrid, (const Acc*)part_a, part_b, cs, tol2,
                                                               next, part_c, kCdotGrid);
      if (co && PupAggOrder<T>::value) {
#define RB_PUP(L_, V_)                                                                                   \
  cg_pupdate_agg_kernel<T, L_, V_><<<agrid, kBlk, 0, st>>>(co->nc, k, cs, dinv, R, P, Xs, co->agg_ptr, \
                                                          co->agg_rows, ec)
        RB_DISPATCH_LV(sh, RB_PUP);
#undef RB_PUP
      } else {
#define RB_PUP(L_, V_) cg_pupdate_kernel<T, L_, V_><<<sh.grid, kBlk, 0, st>>>(n, k, cs, dinv, R, P, Xs, agg, ec)
        RB_DISPATCH_LV(sh, RB_PUP);
#undef RB_PUP
      }
      RB_LAUNCH_CHECK();
      *launches += 5;
      rd ^= 1;
    }
    return RB_OK;
  };
  // Bursts of check_every iterations; the host reads a burst's live count
  // (copied to a snapshot slot at its end) only after it has queued the next
  // burst, so the GPU always has one burst of work queued while the host
  // waits: a host thread that is late by less than a burst's duration costs
  // no GPU time.  The burst queued after the converged one runs as no-ops.
  // With per-kernel timing on, bursts are read one at a time (the timer's
  // events are harvested at each read).
  if (check_every == 0) {
    // fixed budget: every iteration is queued and none is read back; the
    // kernels of iterations after convergence return at once (live == 0)
    RB_TRY(enqueue_burst(maxiter));
    *iters_out = maxiter;
    return RB_OK;
  }
  BurstSync bs;
  RB_TRY(bs.init());
  int it = 0, pend = -1, pend_it = 0, next_snap = 0;
  bool converged = false;
  while (it < maxiter) {
    const int burst = std::min(check_every, maxiter - it);
    RB_TRY(enqueue_burst(burst));
    it += burst;
    RB_CUDA_TRY(cudaMemcpyAsync(snap + next_snap, slot[rd], sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
    RB_CUDA_TRY(cudaEventRecord(bs.ev[next_snap], st));
    if (tm.on) {
      int32_t v = 0;
      RB_TRY(bs.read(next_snap, snap, &v));
      RB_TRY(tm.harvest());
      if (v == 0) {
        converged = true;
        break;
      }
      continue;
    }
    if (pend >= 0) {
      int32_t v = 0;
      RB_TRY(bs.read(pend, snap, &v));
      if (v == 0) {
        converged = true;
        it = pend_it;
        break;
      }
    }
    pend = next_snap;
    pend_it = it;
    next_snap ^= 1;
  }
  (void)converged;
  *iters_out = it;
  return RB_OK;
}

template <typename T64, typename T>
static int solve_block(const rb_csr& A, const double* B, T64* X, int64_t ldx, int64_t k, const rb_solve_opts& o,
                       rb_solve_info& info, SolveBufs<T64, T>& b, const T* val, const T* dinv,
                       const GroupPlan* gp, const RowGroupsDev* rg, const CoarseOp<T>* co, const SegBufs& sb,
                       cudaStream_t st) {
  const int64_t n = A.n;
  const Shape sh = pick_shape(n, k, Bps<T>::value);      // inner (FP32 or FP64) vector kernels
  Shape shs = pick_spmm_shape<T>(n, k);                  // inner SpMM
  if (o.spmm_lanes > 0 && shs.S == 1) {
    // a caller's (autotuner's) lane count per row: V columns per lane so
    // that L V covers k, within the layouts the kernels are built for
    const int L = o.spmm_lanes, V = (int)ceil_div(k, L);
    if ((L == 4 || L == 8 || L == 16 || L == 32) && (V == 1 || V == 2 || V == 4) && k % V == 0) {
      shs.L = L;
      shs.V = V;
      shs.grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(num_sms() * BpsSpmm<T>::value,
                                                                  ceil_div(n, kBlk / L)));
    }
  }
  const Shape sh64 = pick_shape(n, k, BpsSpmm<T64>::value);  // FP64 residual kernels
  const unsigned fg = (unsigned)ceil_div(k, 8);
  const unsigned eg = (unsigned)std::min<int64_t>(ceil_div(n * k, 256), 148 * 16);
  int launches = 0;
  if (ldx != k) return fail(RB_EARG, "solve_block: internal ldx");
  if (!shape_covers(sh, k) || !shape_covers(shs, k) || !shape_covers(sh64, k))
    return fail(RB_EARG, "solve_block: %lld columns not covered by the lane layout", (long long)k);
  // ||b|| per column
#define RB_CN(L_, V_) colnorm_kernel<L_, V_><<<sh64.grid, kBlk, 0, st>>>(n, k, B, b.part_b)
  RB_DISPATCH_LV(sh64, RB_CN);
#undef RB_CN
  RB_LAUNCH_CHECK();
  fin_bnorm_kernel<<<fg, 256, 0, st>>>(k, (int)sh64.grid, b.part_b, b.os);
  if (!o.use_x0) RB_CUDA_TRY(cudaMemsetAsync(X, 0, sizeof(T64) * n * k, st));
  launches += 2;
  const bool segm = sb.in != nullptr;
  const int64_t ninst = segm ? sb.in->ninst : 0, nseg = ninst * k;
  const unsigned sgg = (unsigned)std::min<int64_t>(std::max<int64_t>(ninst, 1), 148 * 8);
  const unsigned sgm = (unsigned)ceil_div(std::max<int64_t>(nseg, 1), 256);
  const int32_t* rinst = segm ? sb.in->row_inst : nullptr;
  const OuterState* scale_state = segm ? sb.seg : b.os;
  if (segm) {
    seg_norm_kernel<double><<<sgg, kSegWarps * 32, 0, st>>>(ninst, k, sb.in->row_ptr, B, sb.s2);
    seg_bnorm_kernel<<<sgm, 256, 0, st>>>(nseg, sb.s2, sb.seg);
    RB_LAUNCH_CHECK();
    launches += 2;
  }
  const double stall = 0.25;
  const bool budget = o.check_every == 0;
  KernelTimer tm;
  tm.on = o.profile != 0 && !budget;
  tm.with_coarse = o.coarse != nullptr;
  int total_iters = 0, outer = 0;
  int sweep_flag = 0;
  for (outer = 0; outer <= o.max_outer; ++outer) {
    // R64 = B - A X (FP64)
    RB_TRY((spmm_t<T64, EPI_RESID>(A, (const T64*)A.val64, X, b.R64, B, b.part_b, k, sh64, st)));
    RB_CUDA_TRY(cudaMemsetAsync(b.counter + 1, 0, sizeof(int32_t), st));
    const double itol_min = sizeof(T) == sizeof(T64) ? o.inner_tol : std::min(o.inner_tol, 1e-6);
    if (segm) {
      seg_norm_kernel<T64><<<sgg, kSegWarps * 32, 0, st>>>(ninst, k, sb.in->row_ptr, b.R64, sb.s2);
      seg_outer_kernel<<<sgm, 256, 0, st>>>(nseg, sb.s2, sb.seg, o.tol, stall, o.inner_tol, itol_min);
      seg_summary_kernel<<<(unsigned)ceil_div(k, 128), 128, 0, st>>>(ninst, k, sb.seg, b.os, b.counter + 1);
      launches += 2;
    } else {
      fin_outer_kernel<<<fg, 256, 0, st>>>(k, (int)sh64.grid, b.part_b, b.os, o.tol, stall, o.inner_tol, itol_min,
                                           b.counter + 1);
    }
    RB_LAUNCH_CHECK();
    launches += 2;
    if (budget) {
      // fixed budget: max_outer sweeps, none read back; a done column's
      // cast, solve and correction are no-ops
      if (outer == o.max_outer) break;
    } else {
      int32_t nact = 0;
      RB_CUDA_TRY(cudaMemcpyAsync(&nact, b.counter + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
      RB_CUDA_TRY(cudaStreamSynchronize(st));
      if (nact == 0 || outer == o.max_outer) break;
    }
    cast_scale_kernel<T64, T><<<eg, 256, 0, st>>>(n, k, b.R64, scale_state, rinst, b.R);
    RB_LAUNCH_CHECK();
    launches += 1;
    int it = 0;
    RB_TRY(inner_solve<T>(A, val, dinv, k, sh, shs, b.part_a, b.part_b, b.Xs, b.R, b.P, b.Q, b.cs, nullptr,
                          b.os, b.counter, o.inner_tol, o.maxiter, o.check_every, &it, &launches, tm, gp, rg,
                          co, st));
    total_iters += it;
    info.sweep_iters_max = std::max(info.sweep_iters_max, it);
    if (it >= o.maxiter) sweep_flag = 1;
    correct_kernel<T64, T><<<eg, 256, 0, st>>>(n, k, b.Xs, scale_state, rinst, X);
    RB_LAUNCH_CHECK();
    launches += 1;
  }
  if (segm) {
    seg_status_kernel<<<(unsigned)ceil_div(ninst, 128), 128, 0, st>>>(ninst, k, sb.ncol, sb.seg, b.cs, b.counter,
                                                                       sb.in->status, sb.in->relres);
    RB_LAUNCH_CHECK();
    launches += 1;
  }
  if (budget) {  // nothing is read back: the outcome is in the status words
    info.iters += outer * o.maxiter;
    info.outer = std::max(info.outer, outer);
    info.flag = -1;
    info.launches += launches;
    info.relres = -1.0;
    return RB_OK;
  }
  // summary
  int32_t hcnt[4] = {0, 0, 0, 0};
  RB_CUDA_TRY(cudaMemcpyAsync(hcnt, b.counter, sizeof(hcnt), cudaMemcpyDeviceToHost, st));
  std::vector<OuterState> hos(k);
  RB_CUDA_TRY(cudaMemcpyAsync(hos.data(), b.os, sizeof(OuterState) * k, cudaMemcpyDeviceToHost, st));
  std::vector<ColState> hcs(k);
  RB_CUDA_TRY(cudaMemcpyAsync(hcs.data(), b.cs, sizeof(ColState) * k, cudaMemcpyDeviceToHost, st));
  RB_CUDA_TRY(cudaStreamSynchronize(st));
  if (hcnt[2]) return fail(RB_ECUDA, "rb_femsolve: SpMM shared-memory copy did not complete in time");
  double worst = 0.0;
  int flag = 0;
  for (int64_t c = 0; c < k; ++c) {
    worst = std::isfinite(hos[c].relres) ? std::max(worst, hos[c].relres) : hos[c].relres;
    if (hos[c].done == 0 || (hos[c].done == 2 && hos[c].relres > 1e-10)) flag = std::max(flag, 1);
    if ((hcs[c].status == 2 && hos[c].relres > 1e-10) || hos[c].done == 3) flag = 2;
  }
  if (flag == 1 && sweep_flag == 0 && worst <= o.tol) flag = 0;
  if (segm) {  // the flag of the worst instance
    std::vector<int32_t> hst(ninst);
    RB_CUDA_TRY(cudaMemcpyAsync(hst.data(), sb.in->status, sizeof(int32_t) * ninst, cudaMemcpyDeviceToHost, st));
    RB_CUDA_TRY(cudaStreamSynchronize(st));
    flag = 0;
    for (int32_t v : hst) flag = std::max(flag, v >= 2 ? 2 : v);
  }
  info.iters += total_iters;
  info.outer = std::max(info.outer, outer);
  info.flag = std::max(info.flag, flag);
  info.launches += launches;
  info.relres = std::max(info.relres, worst);
  info.spmm_ms += tm.spmm_ms;
  info.spmm_launches += tm.spmm_n;
  info.update_ms += tm.upd_ms;
  info.update_launches += tm.upd_n;
  info.coarse_ms += tm.coarse_ms;
  info.coarse_launches += tm.coarse_n;
  return RB_OK;
}

template <typename T64, typename T>
static int femsolve_t(const rb_csr& A, const double* B, T64* X, int64_t nrhs, const rb_solve_opts& o,
                      rb_solve_info& info, void* work, size_t work_bytes, const T* val, const T* dinv,
                      cudaStream_t st) {
  const int64_t n = A.n;
  if (nrhs > kMaxCols) return fail(RB_ESIZE, "rb_femsolve: more than %lld right-hand sides per call", (long long)kMaxCols);
  const int64_t kb = solve_cols(nrhs);  // columns of the solve (padded when the layout needs it)
  Carver cv{reinterpret_cast<char*>(work), work_bytes};
  SolveBufs<T64, T> b;
  carve(cv, b, n, A.nnz, kb);
  if (!b.scan_work) return fail(RB_EARG, "rb_femsolve: workspace too small");
  double* Bp = nullptr;
  T64* Xp = nullptr;
  if (kb != nrhs) {
    Bp = cv.take<double>(n * kb);
    Xp = cv.take<T64>(n * kb);
    if (!Bp || !Xp) return fail(RB_EARG, "rb_femsolve: workspace too small");
  }
  CoarseBufs<T64, T> cb;
  if (o.coarse) {
    cb.op.agg = o.coarse->agg;
    cb.op.agg_ptr = o.coarse->agg_ptr;
    cb.op.agg_rows = o.coarse->agg_rows;
    coarse_carve(cv, cb, o.coarse->nc, kb);
    if (!cb.A64 || !cb.Rb || !cb.Cb || !cb.Dinv || !cb.op.X || !cb.op.rc || !cb.op.ec || !cb.op.part || !cb.err)
      return fail(RB_EARG, "rb_femsolve: workspace too small for the coarse space");
  }
  SegBufs sb;
  if (o.instances) {
    sb.in = o.instances;
    sb.ncol = nrhs;
    seg_carve(cv, sb, o.instances->ninst, kb);
    if (!sb.s2 || !sb.seg) return fail(RB_EARG, "rb_femsolve: workspace too small for the instances");
  }
  RB_CUDA_TRY(cudaMemsetAsync(b.counter, 0, 8 * sizeof(int32_t), st));
  if (o.coarse) {
    RB_TRY((coarse_setup<T64, T>(A, cb, st)));
    info.launches += 3 + 5 * (int)ceil_div(cb.op.nc, kGjB);
  }
  GroupPlan gp{nullptr, nullptr, nullptr, 0};
  // spatial row groups (blocked SpMM) when the caller built them for this
  // pattern and the column count fits; else the row-pair / row-group plans
  RowGroupsDev rgd{0, nullptr, nullptr, nullptr, nullptr, nullptr};
  const rb_rowgroups* og = o.groups;
  const bool use_rg = og && og->ng > 0 && og->rows && og->uptr && og->ucol && og->umask && og->coef &&
                      blk_cols_ok<T>(n, kb);
  if (use_rg) {
    rgd = RowGroupsDev{og->ng, og->rows, og->uptr, og->ucol, og->umask, og->coef};
    RB_TRY(rg_fill_coef<T>(A, val, rgd, st));
    info.launches += 1;
  }
  const bool plan = !use_rg && ((GrpCfg<T>::enabled && grp_cols_ok(kb)) ||
                                (PairCfg<T>::enabled && pair_cols_ok<T>(kb) && n * kb < (int64_t(1) << 31)));
  if (plan && n > 0)
    RB_TRY(build_group_plan<GrpCfg<T>::G>(A, b.gcnt, b.gptr, b.ucol, b.umask, b.scan_work, b.scan_bytes, &gp, st));
  const unsigned eg = (unsigned)std::min<int64_t>(ceil_div(n * kb, 256), 148 * 16);
  if (Bp) {
    copy_cols_kernel<double><<<eg, 256, 0, st>>>(n, nrhs, kb, B, Bp);
    RB_LAUNCH_CHECK();
    if (o.use_x0) {
      copy_cols_kernel<T64><<<eg, 256, 0, st>>>(n, nrhs, kb, X, Xp);
      RB_LAUNCH_CHECK();
    }
  }
  RB_TRY((solve_block<T64, T>(A, Bp ? Bp : B, Xp ? Xp : X, kb, kb, o, info, b, val, dinv, gp.ng ? &gp : nullptr,
                              use_rg ? &rgd : nullptr, o.coarse ? &cb.op : nullptr, sb, st)));
  if (Xp) {
    copy_cols_kernel<T64><<<eg, 256, 0, st>>>(n, kb, nrhs, Xp, X);
    RB_LAUNCH_CHECK();
    info.launches += o.use_x0 ? 3 : 2;
  }
  return RB_OK;
}

// FP32 copy of the values and reciprocal diagonal of a CSR matrix
template <typename T64, typename T32>
__global__ void csr_prepare_kernel(int64_t n, const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
                                   const T64* __restrict__ v64, T32* __restrict__ v32, T64* __restrict__ d64,
                                   T32* __restrict__ d32) {
  for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < n; row += (int64_t)gridDim.x * blockDim.x) {
    T64 dg = s_zero(T64());
    for (int32_t p = indptr[row]; p < indptr[row + 1]; ++p) {
      const T64 v = v64[p];
      if (v32) {
        if constexpr (Scalar<T64>::is_complex) v32[p] = T32{(float)v.x, (float)v.y};
        else v32[p] = (T32)v;
      }
      if (indices[p] == row) dg = s_add(dg, v);
    }
    T64 r;
    if constexpr (Scalar<T64>::is_complex) {
      const double d = dg.x * dg.x + dg.y * dg.y;
      r = make_double2(dg.x / d, -dg.y / d);
    } else {
      r = 1.0 / dg;
    }
    if (d64) d64[row] = r;
    if (d32) {
      if constexpr (Scalar<T64>::is_complex) d32[row] = T32{(float)r.x, (float)r.y};
      else d32[row] = (T32)r;
    }
  }
}

}  // namespace rb

using namespace rb;

extern "C" {

size_t rb_femsolve_work_bytes(int64_t n, int64_t nnz, int64_t nrhs, int32_t is_complex, int32_t precision) {
  const int64_t k0 = std::min<int64_t>(std::max<int64_t>(nrhs, 1), kMaxCols), k = solve_cols(k0);
  Carver cv{nullptr, 0};
  size_t bytes;
  if (is_complex) {
    if (precision == RB_FP64) { SolveBufs<cdouble, cdouble> b; bytes = carve(cv, b, n, nnz, k); }
    else { SolveBufs<cdouble, cfloat> b; bytes = carve(cv, b, n, nnz, k); }
  } else {
    if (precision == RB_FP64) { SolveBufs<double, double> b; bytes = carve(cv, b, n, nnz, k); }
    else { SolveBufs<double, float> b; bytes = carve(cv, b, n, nnz, k); }
  }
  if (k != k0) {  // the padded copies of B and X
    cv.take<double>(n * k);
    if (is_complex) cv.take<cdouble>(n * k);
    else cv.take<double>(n * k);
    bytes = cv.used;
  }
  return bytes + 4096;
}

size_t rb_instances_work_bytes(int64_t ninst, int64_t nrhs) {
  if (ninst < 1) return 0;
  const int64_t k = solve_cols(std::min<int64_t>(std::max<int64_t>(nrhs, 1), kMaxCols));
  Carver cv{nullptr, 0};
  SegBufs sb;
  return seg_carve(cv, sb, ninst, k) + 512;
}

size_t rb_coarse_work_bytes(int64_t nc, int64_t nrhs, int32_t is_complex, int32_t precision) {
  const int64_t k = solve_cols(std::min<int64_t>(std::max<int64_t>(nrhs, 1), kMaxCols));
  Carver cv{nullptr, 0};
  if (nc < 1) return 0;
  if (is_complex) {
    if (precision == RB_FP64) { CoarseBufs<cdouble, cdouble> c; return coarse_carve(cv, c, nc, k); }
    CoarseBufs<cdouble, cfloat> c;
    return coarse_carve(cv, c, nc, k);
  }
  if (precision == RB_FP64) { CoarseBufs<double, double> c; return coarse_carve(cv, c, nc, k); }
  CoarseBufs<double, float> c;
  return coarse_carve(cv, c, nc, k);
}

int rb_femsolve(const rb_csr* A, const double* B, void* X, int64_t nrhs, const rb_solve_opts* opts,
                rb_solve_info* info, void* work, size_t work_bytes, void* stream) {
  if (!A || !B || !X || !opts || !info || !work) return fail(RB_EARG, "rb_femsolve: null argument");
  if (nrhs < 1 || A->n < 1) return fail(RB_EARG, "rb_femsolve: empty system");
  if (nrhs > kMaxCols) return fail(RB_ESIZE, "rb_femsolve: at most %lld right-hand sides per call", (long long)kMaxCols);
  const rb_solve_opts& o = *opts;
  if (o.precision != RB_MIXED && o.precision != RB_FP64) return fail(RB_EARG, "rb_femsolve: bad precision");
  if (!A->val64 || !A->dinv64 || !A->indptr || !A->indices) return fail(RB_EARG, "rb_femsolve: matrix arrays missing");
  if (o.precision == RB_MIXED && (!A->val32 || !A->dinv32)) return fail(RB_EARG, "rb_femsolve: mixed precision needs val32/dinv32");
  if (o.maxiter < 1 || o.check_every < 0 || o.max_outer < 1 || !(o.tol > 0) || !(o.inner_tol > 0))
    return fail(RB_EARG, "rb_femsolve: bad options");
  if (o.check_every == 0 && (!o.instances || o.coarse))
    return fail(RB_EARG, "rb_femsolve: a fixed budget (check_every 0) needs instances (the status words) "
                         "and no coarse space");
  size_t need = rb_femsolve_work_bytes(A->n, A->nnz, nrhs, A->is_complex, o.precision);
  if (o.coarse) {
    const rb_coarse& c = *o.coarse;
    if (c.nc < 1 || c.nc > kCoarseMax || c.nc > A->n || !c.agg || !c.agg_ptr || !c.agg_rows)
      return fail(RB_EARG, "rb_femsolve: coarse space needs 1 <= nc <= min(n, %d) and its three arrays", kCoarseMax);
    need += rb_coarse_work_bytes(c.nc, nrhs, A->is_complex, o.precision);
  }
  if (o.instances) {
    const rb_instances& in = *o.instances;
    if (in.ninst < 1 || !in.row_ptr || !in.row_inst || !in.status)
      return fail(RB_EARG, "rb_femsolve: instances need ninst >= 1, row_ptr, row_inst and status");
    need += rb_instances_work_bytes(in.ninst, nrhs);
  }
  if (work_bytes < need) return fail(RB_EARG, "rb_femsolve: workspace too small");
  *info = rb_solve_info{};
  cudaStream_t st = as_stream(stream);
  if (A->is_complex) {
    if (o.precision == RB_FP64)
      return femsolve_t<cdouble, cdouble>(*A, B, (cdouble*)X, nrhs, o, *info, work, work_bytes,
                                          (const cdouble*)A->val64, (const cdouble*)A->dinv64, st);
    return femsolve_t<cdouble, cfloat>(*A, B, (cdouble*)X, nrhs, o, *info, work, work_bytes,
                                       (const cfloat*)A->val32, (const cfloat*)A->dinv32, st);
  }
  if (o.precision == RB_FP64)
    return femsolve_t<double, double>(*A, B, (double*)X, nrhs, o, *info, work, work_bytes,
                                      (const double*)A->val64, (const double*)A->dinv64, st);
  return femsolve_t<double, float>(*A, B, (double*)X, nrhs, o, *info, work, work_bytes,
                                   (const float*)A->val32, (const float*)A->dinv32, st);
}

int rb_spmm(const rb_csr* A, int32_t kind, const void* X, void* Y, int64_t nrhs, void* stream) {
  if (!A || !X || !Y || nrhs < 1) return fail(RB_EARG, "rb_spmm: bad arguments");
  if (nrhs > kMaxCols) return fail(RB_ESIZE, "rb_spmm: at most %lld columns", (long long)kMaxCols);
  const Shape sh = pick_shape(A->n, nrhs, 3);
  cudaStream_t st = as_stream(stream);
  if (!shape_covers(sh, nrhs)) {
    const unsigned g = (unsigned)std::min<int64_t>(ceil_div(A->n, 8), 148 * 16);
    switch (kind) {
      case RB_F64: spmm_any_kernel<double><<<g, 256, 0, st>>>(A->n, nrhs, A->indptr, A->indices, (const double*)A->val64, (const double*)X, (double*)Y); break;
      case RB_C128: spmm_any_kernel<cdouble><<<g, 256, 0, st>>>(A->n, nrhs, A->indptr, A->indices, (const cdouble*)A->val64, (const cdouble*)X, (cdouble*)Y); break;
      case RB_F32: spmm_any_kernel<float><<<g, 256, 0, st>>>(A->n, nrhs, A->indptr, A->indices, (const float*)A->val32, (const float*)X, (float*)Y); break;
      case RB_C64: spmm_any_kernel<cfloat><<<g, 256, 0, st>>>(A->n, nrhs, A->indptr, A->indices, (const cfloat*)A->val32, (const cfloat*)X, (cfloat*)Y); break;
      default: return fail(RB_EARG, "rb_spmm: bad kind");
    }
    RB_LAUNCH_CHECK();
    return RB_OK;
  }
  switch (kind) {
    case RB_F64: return spmm_t<double, EPI_STORE>(*A, (const double*)A->val64, (const double*)X, (double*)Y, nullptr, nullptr, nrhs, sh, st);
    case RB_C128: return spmm_t<cdouble, EPI_STORE>(*A, (const cdouble*)A->val64, (const cdouble*)X, (cdouble*)Y, nullptr, nullptr, nrhs, sh, st);
    case RB_F32: return spmm_t<float, EPI_STORE>(*A, (const float*)A->val32, (const float*)X, (float*)Y, nullptr, nullptr, nrhs, sh, st);
    case RB_C64: return spmm_t<cfloat, EPI_STORE>(*A, (const cfloat*)A->val32, (const cfloat*)X, (cfloat*)Y, nullptr, nullptr, nrhs, sh, st);
    default: return fail(RB_EARG, "rb_spmm: bad kind");
  }
}

int rb_csr_prepare(const rb_csr* A, void* val32, void* dinv64, void* dinv32, void* stream) {
  if (!A || !A->indptr || !A->indices || !A->val64 || A->n < 1) return fail(RB_EARG, "rb_csr_prepare: bad matrix");
  const unsigned g = (unsigned)std::min<int64_t>(ceil_div(A->n, 256), 148 * 16);
  cudaStream_t st = as_stream(stream);
  if (A->is_complex)
    csr_prepare_kernel<cdouble, cfloat><<<g, 256, 0, st>>>(A->n, A->indptr, A->indices, (const cdouble*)A->val64,
                                                           (cfloat*)val32, (cdouble*)dinv64, (cfloat*)dinv32);
  else
    csr_prepare_kernel<double, float><<<g, 256, 0, st>>>(A->n, A->indptr, A->indices, (const double*)A->val64,
                                                         (float*)val32, (double*)dinv64, (float*)dinv32);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

}  // extern "C"
