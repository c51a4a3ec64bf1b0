// Blocked SpMM over spatial row groups (included by rb_krylov.cu).
//
// A group is up to kRG = 8 rows that sit close together in the mesh (built by
// rb_rowgroups_bin: the nodes of one cube of edge ~2 node spacings, i.e. a
// 2 x 2 x 2 block on a structured grid).  The union of the group's column
// lists (ascending, each entry with an 8-bit mask of the rows holding it) is
// built once per pattern; per matrix the coefficients are laid out per union
// entry as kRG values (0 where a row lacks the column), so one warp walks the
// union once, gathers each x row ONCE for all eight rows and applies it from
// registers (packed FP32x2 FMAs, each row's sum in ascending column order:
// the same bits as the per-row kernels).  On the tetrahedral box a 2 x 2 x 2
// group needs 5.7 x rows per matrix row against 14.2 nonzeros (10.5 for the
// row-pair kernel); L2 -> SM traffic drops from 2.13 to 1.38 GB per
// 128-column product and the kernel runs 210 us against 229 us on the
// 3M-tet box: the gathers are bounded by the misses an SM keeps in flight,
// not by their count (measured: the same kernel without its FMAs takes
// 175 us; with x resident in L2 the time per row is unchanged), so the
// occupancy that holds the most warps gathering at once wins.
//
// Lane layout: lane l owns columns [4 l, 4 l + 4).
#pragma once

namespace rb {

constexpr int kRG = 8;  // rows per spatial group

struct RowGroupsDev {
  int64_t ng;
  const int32_t* rows;   // ng x kRG, -1 pads
  const int32_t* uptr;   // ng + 1
  const int32_t* ucol;   // nu
  const uint8_t* umask;  // nu
  void* coef;            // nu x kRG values of the solve's FP32 kind
};

// coefficient table of one matrix: coef[u][r] = A[rows[r], ucol[u]] or 0
template <typename T>
__global__ void rg_coef_kernel(int64_t ng, const int32_t* __restrict__ rows, const int32_t* __restrict__ uptr,
                               const int32_t* __restrict__ ucol, const int32_t* __restrict__ indptr,
                               const int32_t* __restrict__ indices, const T* __restrict__ val,
                               T* __restrict__ coef) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < ng; g += (int64_t)gridDim.x * blockDim.x) {
    int32_t p[kRG], e[kRG];
#pragma unroll
    for (int r = 0; r < kRG; ++r) {
      const int32_t row = rows[g * kRG + r];
      p[r] = row >= 0 ? indptr[row] : 0;
      e[r] = row >= 0 ? indptr[row + 1] : 0;
    }
    const int32_t ue = uptr[g + 1];
    for (int32_t u = uptr[g]; u < ue; ++u) {
      const int32_t c = ucol[u];
      T a[kRG];
#pragma unroll
      for (int r = 0; r < kRG; ++r) {
        a[r] = s_zero(T());
        if (p[r] < e[r] && indices[p[r]] == c) a[r] = val[p[r]++];
      }
#pragma unroll
      for (int r = 0; r < kRG; ++r) coef[(int64_t)u * kRG + r] = a[r];
    }
  }
}

template <typename T> struct BlkOn { static constexpr bool value = std::is_same<T, float>::value; };
template <typename T> struct BlkCfg;
// FP32: 128 columns as 32 lanes x 4
// U = 4 gathers in flight per warp at 3 blocks per SM (80 registers) beat
// U = 8 at 2 blocks (118 registers): 0.210 against 0.221 ms on the 3M-tet box;
// U = 2 at 4 blocks spills (0.229 ms)
template <> struct BlkCfg<float> {
  static constexpr int V = 4, U = 4, BPS = 3;
};

template <typename T> static bool blk_cols_ok(int64_t n, int64_t k) {
  if constexpr (std::is_same<T, float>::value) return k > 64 && k <= 128 && k % 4 == 0 && n * k < (int64_t(1) << 31);
  return false;
}

// q = A p for the group's rows plus the fused p.q column sums (EPI_PQDOT),
// x rows gathered from global memory into registers.
template <typename T>
__global__ void __launch_bounds__(kBlk, BlkCfg<T>::BPS)
spmm_blk_kernel(int64_t k, RowGroupsDev rg, const T* __restrict__ X, T* __restrict__ Y, void* __restrict__ part_,
                const int32_t* __restrict__ live) {
  if (live && *live == 0) return;  // every column converged: a no-op iteration
  constexpr int V = BlkCfg<T>::V, U = BlkCfg<T>::U;
  typedef typename Scalar<T>::acc A;
  constexpr int W = kBlk / 32;
  constexpr int NP = kRG / 2;
  __shared__ A sm[kBlk * V];
  __shared__ __align__(16) int32_t s_off[W][32];
  __shared__ __align__(16) uint8_t s_pm[W][32];
  __shared__ __align__(16) T s_cf[W][32 * kRG];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t task0 = blockIdx.x * (int64_t)W + wid;
  const int64_t c0 = (int64_t)lane * V;
  const bool on = c0 < k;
  const int64_t tasks = (int64_t)gridDim.x * W;
  const T* const xl = X + c0;
  const T* const cf_g = reinterpret_cast<const T*>(rg.coef);
  alignas(16) A acc[V];
#pragma unroll
  for (int j = 0; j < V; ++j) acc[j] = acc_zero<A>();
  for (int64_t g = task0; g < rg.ng; g += tasks) {
    const int32_t myrow = lane < kRG ? rg.rows[g * kRG + lane] : -1;
    const int32_t ub = rg.uptr[g], ue = rg.uptr[g + 1];
    // accumulators of row pair p, column q: (row 2p, row 2p + 1)
    float2 yp[NP][V];
#pragma unroll
    for (int p = 0; p < NP; ++p)
#pragma unroll
      for (int q = 0; q < V; ++q) yp[p][q] = make_float2(0.f, 0.f);
    for (int32_t u0 = ub; u0 < ue; u0 += 32) {
      const int cnt = min(32, ue - u0);
      const int cntp = (cnt + U - 1) / U * U;
      // stage the chunk: x row offsets, pair masks, coefficients (padding
      // entries repeat the last offset at coefficient 0 with an empty mask)
      if (lane < cntp) {
        const bool in = lane < cnt;
        const int32_t u = u0 + min(lane, cnt - 1);
        s_off[wid][lane] = rg.ucol[u] * (int32_t)k;
        const uint32_t m = in ? rg.umask[u] : 0u;
        uint32_t pm = 0;
#pragma unroll
        for (int p = 0; p < NP; ++p) pm |= ((m >> (2 * p)) & 3u) ? (1u << p) : 0u;
        s_pm[wid][lane] = (uint8_t)pm;
        alignas(16) T a[kRG];
        if (in) {
          ldv<T, kRG>(cf_g + (int64_t)u * kRG, a);
        } else {
#pragma unroll
          for (int r = 0; r < kRG; ++r) a[r] = s_zero(T());
        }
        stv<T, kRG>(&s_cf[wid][lane * kRG], a);
      }
      __syncwarp();
      for (int j = 0; j < cntp; j += U) {
        alignas(16) int32_t oo[U];
        ldv_s<int32_t, U>(&s_off[wid][j], oo);
        uint8_t pmv[U];
        if constexpr (U == 8) {
          alignas(8) uint8_t t8[8];
          *reinterpret_cast<uint2*>(t8) = *reinterpret_cast<const uint2*>(&s_pm[wid][j]);
#pragma unroll
          for (int u = 0; u < 8; ++u) pmv[u] = t8[u];
        } else if constexpr (U == 4) {
          const uint32_t w4 = *reinterpret_cast<const uint32_t*>(&s_pm[wid][j]);
#pragma unroll
          for (int u = 0; u < 4; ++u) pmv[u] = (uint8_t)(w4 >> (8 * u));
        } else {
#pragma unroll
          for (int u = 0; u < U; ++u) pmv[u] = s_pm[wid][j + u];
        }
        if (on) {
          alignas(16) T xv[U][V];
#pragma unroll
          for (int u = 0; u < U; ++u) ldv<T, V>(xl + (uint32_t)oo[u], xv[u]);
#pragma unroll
          for (int u = 0; u < U; ++u) {
            alignas(16) float2 ap[NP];
            ldv_s<float2, NP>(reinterpret_cast<const float2*>(&s_cf[wid][(j + u) * kRG]), ap);
            float2 xd[V];
#pragma unroll
            for (int q = 0; q < V; ++q) xd[q] = make_float2(xv[u][q], xv[u][q]);
            const uint32_t pm = pmv[u];
#pragma unroll
            for (int p = 0; p < NP; ++p)
              if (pm & (1u << p)) {
#pragma unroll
                for (int q = 0; q < V; ++q) yp[p][q] = __ffma2_rn(ap[p], xd[q], yp[p][q]);
              }
          }
        }
      }
      __syncwarp();  // the slot is rewritten by the next chunk
    }
#pragma unroll
    for (int r = 0; r < kRG; ++r) {
      const int32_t row = __shfl_sync(0xffffffffu, myrow, r);
      if (on && row >= 0) {
        alignas(16) T pv[V], yv[V];
#pragma unroll
        for (int q = 0; q < V; ++q) yv[q] = (r & 1) ? yp[r / 2][q].y : yp[r / 2][q].x;
        ldv<T, V>(X + (int64_t)row * k + c0, pv);
#pragma unroll
        for (int q = 0; q < V; ++q) acc[q] = acc_fma(pv[q], yv[q], acc[q]);
        stv<T, V>(Y + (int64_t)row * k + c0, yv);
      }
    }
  }
  block_colreduce<A, 32, V, 1>(acc, reinterpret_cast<A*>(part_), k, sm);
}

template <typename T>
static int spmm_blk(const RowGroupsDev& rg, const T* X, T* Y, void* part, int64_t k, unsigned* grid_out,
                    cudaStream_t st, const int32_t* live) {
  const unsigned grid = (unsigned)std::max<int64_t>(
      1, std::min<int64_t>(num_sms() * BlkCfg<T>::BPS, ceil_div(rg.ng, kBlk / 32)));
  spmm_blk_kernel<T><<<grid, kBlk, 0, st>>>(k, rg, X, Y, part, live);
  RB_LAUNCH_CHECK();
  *grid_out = grid;
  return RB_OK;
}

template <typename T>
static int rg_fill_coef(const rb_csr& A, const T* val, const RowGroupsDev& rg, cudaStream_t st) {
  if (rg.ng == 0) return RB_OK;
  const unsigned grid = (unsigned)std::min<int64_t>(ceil_div(rg.ng, 128), 148 * 16);
  rg_coef_kernel<T><<<grid, 128, 0, st>>>(rg.ng, rg.rows, rg.uptr, rg.ucol, A.indptr, A.indices, val,
                                          reinterpret_cast<T*>(rg.coef));
  RB_LAUNCH_CHECK();
  return RB_OK;
}

}  // namespace rb
