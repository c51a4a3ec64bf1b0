// FEM matrix assembly (femlhs) into a fixed CSR pattern.
//
// The geometry of a mesh is fixed across Gauss-Newton iterations, so its
// per-tet gradient products (deldotdel, ne x 10) and volumes are computed
// once by rb_deldotdel; every assembly then only combines them with the
// current optical properties, as redbirdpy's femlhs does with cfg['deldotdel'].
//
// One warp owns one matrix row n.  Its lanes first evaluate, for up to 32
// tets that contain n, the tet's contribution to row n (4 values: row li of
// the local 4x4 block D_e*K_e + mass(mua) (+ i*omega/c*mass(n))) and stage
// them in shared memory.  The lanes then switch roles and each owns one CSR
// slot of the row, summing the staged contributions whose column matches in
// ascending tet order, then the Robin terms of the row's boundary faces.  No
// atomics: the result is deterministic and written exactly once (FP64 plus an
// optional FP32 copy), together with the reciprocal diagonal used by the
// Jacobi preconditioner.  A prologue pass stores the diffusion coefficient
// D = 1/(3(mua+musp)) per node (or per tet) in the workspace so that no
// division is repeated per incidence.
#include <algorithm>
#include <mutex>

#include "rb_common.cuh"

namespace rb {

constexpr int kAsmWarps = 8;

template <bool CPLX> struct AsmVal;
template <> struct AsmVal<false> { typedef double T; typedef float T32; };
template <> struct AsmVal<true> { typedef cdouble T; typedef cfloat T32; };

__device__ __forceinline__ void put(double& dst, double re, double) { dst = re; }
__device__ __forceinline__ void put(cdouble& dst, double re, double im) { dst = make_double2(re, im); }
__device__ __forceinline__ float narrow(double v) { return (float)v; }
__device__ __forceinline__ cfloat narrow(cdouble v) { return make_float2((float)v.x, (float)v.y); }
__device__ __forceinline__ double recip(double v) { return 1.0 / v; }
__device__ __forceinline__ cdouble recip(cdouble v) {
  const double d = v.x * v.x + v.y * v.y;
  return make_double2(v.x / d, -v.y / d);
}
__device__ __forceinline__ void add_real(double& a, double v) { a += v; }
__device__ __forceinline__ void add_real(cdouble& a, double v) { a.x += v; }

__global__ void dcoeff_kernel(int64_t m, const double* __restrict__ mua, const double* __restrict__ musp,
                              double* __restrict__ dco) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
    dco[i] = 1.0 / (3.0 * (mua[i] + musp[i]));
}

// deldotdel column of the pair (a, b), a, b in 0..3
__device__ __forceinline__ int ddd_col(int a, int b) {
  const int lo = a < b ? a : b, hi = a < b ? b : a;
  return lo * 4 - (lo * (lo - 1)) / 2 + (hi - lo);
}

// Contribution of tet `e` (nodes en) to row `row`: the 4 entries (row, en[j]).
template <bool CPLX, int KIND>
__device__ __forceinline__ void tet_row(const rb_mesh& m, const rb_optics& o, const double* __restrict__ evol,
                                        const double* __restrict__ ddd, const double* __restrict__ dco, double wc,
                                        int64_t e, int4 en, int64_t row, typename AsmVal<CPLX>::T out[4]) {
  const int li = (en.y == row) ? 1 : (en.z == row) ? 2 : (en.w == row) ? 3 : 0;
  const double vol = evol[e];
  const double* dd = ddd + 10 * e;
  double k4[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) k4[j] = dd[ddd_col(li, j)];
  double d_e, mu[4], nr[4];
  double msum = 0.0, nsum = 0.0, mli = 0.0, nli = 0.0;
  const bool nvec = (o.nref != nullptr);
  const int32_t nd[4] = {en.x, en.y, en.z, en.w};
  if (KIND == RB_PROP_NODE) {
    double ds = 0.0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      mu[j] = o.mua[nd[j]];
      msum += mu[j];
      ds += dco[nd[j]];
      nr[j] = nvec ? o.nref[nd[j]] : o.nref_scalar;
      nsum += nr[j];
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (j == li) {
        mli = mu[j];
        nli = nr[j];
      }
    }
    d_e = 0.25 * ds;
  } else {
    d_e = dco[e];
    const double ma = o.mua[e], ne_ = nvec ? o.nref[e] : o.nref_scalar;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      mu[j] = ma;
      nr[j] = ne_;
    }
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const double stiff = d_e * k4[j];
    const bool dg = (j == li);
    double mass, imag = 0.0;
    if (KIND == RB_PROP_NODE) {
      // lumped-weight mass of node-based properties (femlhs w1/w2):
      // (sum + mu_i + mu_j)/120 off the diagonal, (sum + 2 mu_i)/60 on it
      mass = dg ? vol * (msum + 2.0 * mli) * (1.0 / 60.0) : vol * (msum + mli + mu[j]) * (1.0 / 120.0);
      if (CPLX) {
        if (nvec)
          imag = dg ? wc * vol * (nsum + 2.0 * nli) * (1.0 / 60.0)
                    : wc * vol * (nsum + nli + nr[j]) * (1.0 / 120.0);
        else
          imag = wc * o.nref_scalar * (dg ? 0.10 : 0.05) * vol;
      }
    } else {
      mass = (dg ? 0.10 : 0.05) * mu[0] * vol;
      if (CPLX) imag = (dg ? 0.10 : 0.05) * wc * nr[0] * vol;
    }
    put(out[j], stiff + mass, imag);
  }
}

template <bool CPLX, int KIND>
__global__ void __launch_bounds__(kAsmWarps * 32)
femlhs_rows_kernel(rb_mesh m, rb_optics o, const double* __restrict__ evol, const double* __restrict__ ddd,
                   const double* __restrict__ dco, double bc, double wc,
                   typename AsmVal<CPLX>::T* __restrict__ val64, typename AsmVal<CPLX>::T32* __restrict__ val32,
                   typename AsmVal<CPLX>::T* __restrict__ dinv64, typename AsmVal<CPLX>::T32* __restrict__ dinv32) {
  typedef typename AsmVal<CPLX>::T T;
  __shared__ int4 s_nodes[kAsmWarps][32];
  __shared__ T s_vals[kAsmWarps][32][4];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t warps = (int64_t)gridDim.x * kAsmWarps;
  for (int64_t row = blockIdx.x * (int64_t)kAsmWarps + w; row < m.nn; row += warps) {
    const int32_t rb = m.indptr[row], rn = m.indptr[row + 1] - rb;
    const int32_t eb = m.node_eptr[row], ek = m.node_eptr[row + 1] - eb;
    const int32_t fb = m.node_fptr[row], fk = m.node_fptr[row + 1] - fb;
    for (int32_t sb = 0; sb < rn; sb += 64) {
      const int32_t p0 = sb + lane, p1 = sb + 32 + lane;
      const int32_t col0 = (p0 < rn) ? m.indices[rb + p0] : -1;
      const int32_t col1 = (p1 < rn) ? m.indices[rb + p1] : -1;
      T acc0 = s_zero(T()), acc1 = s_zero(T());
      for (int32_t t0 = 0; t0 < ek; t0 += 32) {
        const int32_t kc = min(32, ek - t0);
        if (lane < kc) {
          const int64_t e = m.node_elist[eb + t0 + lane];
          const int4 en = reinterpret_cast<const int4*>(m.elem)[e];
          T v[4];
          tet_row<CPLX, KIND>(m, o, evol, ddd, dco, wc, e, en, row, v);
          s_nodes[w][lane] = en;
#pragma unroll
          for (int j = 0; j < 4; ++j) s_vals[w][lane][j] = v[j];
        }
        __syncwarp();
        for (int u = 0; u < kc; ++u) {
          const int4 en = s_nodes[w][u];
          if (en.x == col0) acc0 = s_add(acc0, s_vals[w][u][0]);
          if (en.y == col0) acc0 = s_add(acc0, s_vals[w][u][1]);
          if (en.z == col0) acc0 = s_add(acc0, s_vals[w][u][2]);
          if (en.w == col0) acc0 = s_add(acc0, s_vals[w][u][3]);
          if (col1 >= 0) {
            if (en.x == col1) acc1 = s_add(acc1, s_vals[w][u][0]);
            if (en.y == col1) acc1 = s_add(acc1, s_vals[w][u][1]);
            if (en.z == col1) acc1 = s_add(acc1, s_vals[w][u][2]);
            if (en.w == col1) acc1 = s_add(acc1, s_vals[w][u][3]);
          }
        }
        __syncwarp();
      }
      // Robin boundary: area*bc on the diagonal, half of it off the diagonal
      for (int32_t t = 0; t < fk; ++t) {
        const int32_t f = m.node_flist[fb + t];
        const double a = m.area[f] * bc;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const int32_t nq = m.face[3 * (int64_t)f + q];
          const double v = (nq == row) ? a : 0.5 * a;
          if (nq == col0) add_real(acc0, v);
          if (nq == col1) add_real(acc1, v);
        }
      }
      if (col0 >= 0) {
        val64[rb + p0] = acc0;
        if (val32) val32[rb + p0] = narrow(acc0);
        if (col0 == row) {
          const T r = recip(acc0);
          if (dinv64) dinv64[row] = r;
          if (dinv32) dinv32[row] = narrow(r);
        }
      }
      if (col1 >= 0) {
        val64[rb + p1] = acc1;
        if (val32) val32[rb + p1] = narrow(acc1);
        if (col1 == row) {
          const T r = recip(acc1);
          if (dinv64) dinv64[row] = r;
          if (dinv32) dinv32[row] = narrow(r);
        }
      }
    }
  }
}

// Precomputed incidence tables (rb_assembly_tables): for each row n and each
// of its incident tets u (u < 32, ascending), the CSR slots of the tet's 4
// nodes within row n (one byte each), and for each CSR slot the mask of the
// incident tets that hold its column.  With them a slot's sum visits only
// its own contributors (in ascending tet order) instead of comparing every
// staged tet's 4 nodes against its column, and the diagonal (every tet of the
// row contributes) is a fixed-order butterfly sum across the lanes.
__global__ void asm_tables_kernel(rb_mesh m, uint32_t* __restrict__ inc_slot, uint32_t* __restrict__ slot_mask,
                                  int32_t* __restrict__ bad) {
  __shared__ uint32_t s_mask[kAsmWarps][256];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t warps = (int64_t)gridDim.x * kAsmWarps;
  for (int64_t row = blockIdx.x * (int64_t)kAsmWarps + w; row < m.nn; row += warps) {
    const int32_t rb = m.indptr[row], rn = m.indptr[row + 1] - rb;
    const int32_t eb = m.node_eptr[row], ek = m.node_eptr[row + 1] - eb;
    if (ek > 32 || rn > 255) {
      if (lane == 0) atomicExch(bad, 1);
      continue;
    }
    for (int s = lane; s < rn; s += 32) s_mask[w][s] = 0u;
    __syncwarp();
    if (lane < ek) {
      const int4 en = reinterpret_cast<const int4*>(m.elem)[m.node_elist[eb + lane]];
      const int32_t nd[4] = {en.x, en.y, en.z, en.w};
      uint32_t packed = 0;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int lo = 0, hi = rn - 1, pos = 0;
        while (lo <= hi) {  // the column is in the row (the pattern holds every tet's nodes)
          const int mid = (lo + hi) >> 1;
          const int32_t c = m.indices[rb + mid];
          if (c == nd[j]) {
            pos = mid;
            break;
          }
          if (c < nd[j]) lo = mid + 1;
          else hi = mid - 1;
        }
        packed |= (uint32_t)pos << (8 * j);
        atomicOr(&s_mask[w][pos], 1u << lane);
      }
      inc_slot[eb + lane] = packed;
    }
    __syncwarp();
    for (int s = lane; s < rn; s += 32) slot_mask[rb + s] = s_mask[w][s];
    __syncwarp();
  }
}

__device__ __forceinline__ double shfl_xor_s(double v, int o) { return __shfl_xor_sync(0xffffffffu, v, o); }
__device__ __forceinline__ cdouble shfl_xor_s(cdouble v, int o) {
  return make_double2(__shfl_xor_sync(0xffffffffu, v.x, o), __shfl_xor_sync(0xffffffffu, v.y, o));
}

// Table-driven assembly.  A warp holds R rows at once, L = 32 / R lanes per
// row; lane l of a row evaluates its incident tets l, l + L, ... (at most
// 32 / L of them, a row having at most 32 when the tables exist) and stages
// each tet's 4 values for the row in shared memory, so that R x (32 / L)
// independent load chains are in flight per warp.  The diagonal (every tet
// contributes its (li, li) value) is a butterfly sum across the row's lanes;
// then lane l owns CSR slots l, l + L, ... of its row and sums the staged
// values of the tets in the slot's contributor mask in ascending tet order.
// The slot's column index and mask are loaded before the tets, so that their
// latency overlaps the tet loads.
template <bool CPLX, int KIND, int R>
__global__ void __launch_bounds__(kAsmWarps * 32)
femlhs_tab_kernel(rb_mesh m, rb_optics o, const double* __restrict__ evol, const double* __restrict__ ddd,
                  const double* __restrict__ dco, const uint32_t* __restrict__ inc_slot,
                  const uint32_t* __restrict__ slot_mask, double bc, double wc,
                  typename AsmVal<CPLX>::T* __restrict__ val64, typename AsmVal<CPLX>::T32* __restrict__ val32,
                  typename AsmVal<CPLX>::T* __restrict__ dinv64, typename AsmVal<CPLX>::T32* __restrict__ dinv32) {
  typedef typename AsmVal<CPLX>::T T;
  constexpr int L = 32 / R;  // lanes per row
  __shared__ T s_vals[kAsmWarps][R][32][4];
  __shared__ uint32_t s_ps[kAsmWarps][R][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, h = lane / L, j = lane % L;
  const int64_t warps = (int64_t)gridDim.x * kAsmWarps;
  for (int64_t grp = blockIdx.x * (int64_t)kAsmWarps + w; grp * R < m.nn; grp += warps) {
    const int64_t row = grp * R + h;
    int32_t rb = 0, rn = 0, eb = 0, ek = 0, fb = 0, fk = 0;
    if (row < m.nn) {
      rb = m.indptr[row];
      rn = m.indptr[row + 1] - rb;
      eb = m.node_eptr[row];
      ek = m.node_eptr[row + 1] - eb;
      fb = m.node_fptr[row];
      fk = m.node_fptr[row + 1] - fb;
    }
    const int32_t col0 = (j < rn) ? m.indices[rb + j] : -1;
    const uint32_t msk0 = (j < rn) ? slot_mask[rb + j] : 0u;
    int64_t e[R];
    uint32_t ps[R];
    int4 en[R];
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int u = j + L * i;
      e[i] = (u < ek) ? m.node_elist[eb + u] : 0;
      ps[i] = (u < ek) ? inc_slot[eb + u] : 0u;
    }
#pragma unroll
    for (int i = 0; i < R; ++i) en[i] = reinterpret_cast<const int4*>(m.elem)[e[i]];
    T d = s_zero(T());
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int u = j + L * i;
      if (u < ek) {
        T v[4];
        tet_row<CPLX, KIND>(m, o, evol, ddd, dco, wc, e[i], en[i], row, v);
        const int li = (en[i].y == row) ? 1 : (en[i].z == row) ? 2 : (en[i].w == row) ? 3 : 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          s_vals[w][h][u][q] = v[q];
          if (q == li) d = s_add(d, v[q]);
        }
        s_ps[w][h][u] = ps[i];
      }
    }
    // diagonal: butterfly over the row's lanes (offsets below L stay in them)
#pragma unroll
    for (int off = L / 2; off > 0; off >>= 1) d = s_add(d, shfl_xor_s(d, off));
    __syncwarp();
    for (int32_t sl = j; sl < rn; sl += L) {
      const int32_t col = (sl == j) ? col0 : m.indices[rb + sl];
      T acc = s_zero(T());
      if (col == row) {
        acc = d;
      } else {
        uint32_t msk = (sl == j) ? msk0 : slot_mask[rb + sl];
        while (msk) {
          const int u = __ffs(msk) - 1;
          msk &= msk - 1;
          const uint32_t p = s_ps[w][h][u];
          const int q = ((p & 255u) == (uint32_t)sl) ? 0 : (((p >> 8) & 255u) == (uint32_t)sl) ? 1
                        : (((p >> 16) & 255u) == (uint32_t)sl) ? 2 : 3;
          acc = s_add(acc, s_vals[w][h][u][q]);
        }
      }
      // Robin boundary: area*bc on the diagonal, half of it off the diagonal
      for (int32_t t = 0; t < fk; ++t) {
        const int32_t f = m.node_flist[fb + t];
        const double a = m.area[f] * bc;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const int32_t nq = m.face[3 * (int64_t)f + q];
          if (nq == col) add_real(acc, (nq == row) ? a : 0.5 * a);
        }
      }
      val64[rb + sl] = acc;
      if (val32) val32[rb + sl] = narrow(acc);
      if (col == row) {
        const T r = recip(acc);
        if (dinv64) dinv64[row] = r;
        if (dinv32) dinv32[row] = narrow(r);
      }
    }
    __syncwarp();  // the staged values are rewritten for the next rows
  }
}

// rows per warp of the table-driven assembly (measured on the 3M-tet box,
// one pass of the grid: 1 row 0.37 ms, 2 rows 0.29 ms at CW; 4 rows do not
// fit the complex kernel's staging in 48 KB of static shared memory)
constexpr int kTabRowsPerWarp = 2;

template <bool CPLX, int KIND>
int launch_femlhs(const rb_mesh& m, const rb_optics& o, const double* evol, const double* ddd, double* dco,
                  void* v64, void* v32, void* d64, void* d32, cudaStream_t st) {
  typedef typename AsmVal<CPLX>::T T;
  typedef typename AsmVal<CPLX>::T32 T32;
  const double bc = (1.0 - o.reff) / (12.0 * (1.0 + o.reff));
  const double wc = o.omega / kC0;
  const int64_t np = (KIND == RB_PROP_NODE) ? m.nn : m.ne;
  dcoeff_kernel<<<(unsigned)std::min<int64_t>(ceil_div(np, 256), 148 * 16), 256, 0, st>>>(np, o.mua, o.musp, dco);
  RB_LAUNCH_CHECK();
  unsigned g = (unsigned)std::min<int64_t>(ceil_div(m.nn, kAsmWarps), 148 * 64);
  if (m.inc_slot && m.slot_mask) {
    // one pass of the grid over the rows, in row order: the tets a row shares
    // with the rows a grid plane away are then still in L2 when those come
    constexpr int R = kTabRowsPerWarp;
    const unsigned g2 = (unsigned)ceil_div(ceil_div(m.nn, R), kAsmWarps);
    femlhs_tab_kernel<CPLX, KIND, R><<<g2, kAsmWarps * 32, 0, st>>>(m, o, evol, ddd, dco, m.inc_slot, m.slot_mask,
                                                                      bc, wc, (T*)v64, (T32*)v32, (T*)d64,
                                                                      (T32*)d32);
  } else
    femlhs_rows_kernel<CPLX, KIND><<<g, kAsmWarps * 32, 0, st>>>(m, o, evol, ddd, dco, bc, wc, (T*)v64, (T32*)v32,
                                                                   (T*)d64, (T32*)d32);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

}  // namespace rb

using namespace rb;

extern "C" int rb_assembly_tables(const rb_mesh* mesh, uint32_t* inc_slot, uint32_t* slot_mask, int32_t* usable,
                                  void* stream) {
  if (!mesh || !inc_slot || !slot_mask || !usable || mesh->nn < 1)
    return fail(RB_EARG, "rb_assembly_tables: bad arguments");
  const rb_mesh& m = *mesh;
  if (!m.elem || !m.indptr || !m.indices || !m.node_eptr || !m.node_elist)
    return fail(RB_EARG, "rb_assembly_tables: mesh arrays missing");
  cudaStream_t st = as_stream(stream);
  int32_t* bad = nullptr;
  RB_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&bad), sizeof(int32_t), st));
  RB_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int32_t), st));
  unsigned g = (unsigned)std::min<int64_t>(ceil_div(m.nn, kAsmWarps), 148 * 64);
  asm_tables_kernel<<<g, kAsmWarps * 32, 0, st>>>(m, inc_slot, slot_mask, bad);
  const cudaError_t le = cudaGetLastError();
  int32_t hb = 1;
  const cudaError_t ce = cudaMemcpyAsync(&hb, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(bad, st);
  RB_CUDA_TRY(le);
  RB_CUDA_TRY(ce);
  RB_CUDA_TRY(cudaStreamSynchronize(st));
  *usable = hb == 0;
  return RB_OK;
}

extern "C" size_t rb_femlhs_work_bytes(int64_t nn, int64_t ne) {
  return (size_t)std::max(nn, ne) * sizeof(double) + 256;
}

extern "C" int rb_femlhs(const rb_mesh* mesh, const rb_optics* optics, const double* evol, const double* ddd,
                         void* val64, void* val32, void* dinv64, void* dinv32, void* work, size_t work_bytes,
                         void* stream) {
  if (!mesh || !optics || !val64 || !evol || !ddd || !work)
    return fail(RB_EARG, "rb_femlhs: mesh, optics, evol, ddd, val64 and work are required");
  const rb_mesh& m = *mesh;
  const rb_optics& o = *optics;
  if (!m.elem || !m.indptr || !m.indices || !m.node_eptr || !m.node_elist || !m.node_fptr)
    return fail(RB_EARG, "rb_femlhs: mesh arrays missing");
  if (m.nf > 0 && (!m.face || !m.area || !m.node_flist)) return fail(RB_EARG, "rb_femlhs: boundary arrays missing");
  if (!o.mua || !o.musp) return fail(RB_EARG, "rb_femlhs: mua and musp are required");
  if (o.kind != RB_PROP_NODE && o.kind != RB_PROP_ELEM) return fail(RB_EARG, "rb_femlhs: bad property kind");
  if (!(o.omega >= 0.0)) return fail(RB_EARG, "rb_femlhs: omega must be >= 0");
  if (m.nn < 1 || (o.kind == RB_PROP_NODE ? m.nn : m.ne) < 1)
    return fail(RB_EARG, "rb_femlhs: empty mesh (%lld nodes, %lld tets)", (long long)m.nn, (long long)m.ne);
  if (work_bytes < rb_femlhs_work_bytes(m.nn, m.ne)) return fail(RB_EARG, "rb_femlhs: workspace too small");
  cudaStream_t st = as_stream(stream);
  double* dco = reinterpret_cast<double*>(work);
  const bool cplx = o.omega > 0.0;
  if (cplx)
    return o.kind == RB_PROP_NODE
               ? launch_femlhs<true, RB_PROP_NODE>(m, o, evol, ddd, dco, val64, val32, dinv64, dinv32, st)
               : launch_femlhs<true, RB_PROP_ELEM>(m, o, evol, ddd, dco, val64, val32, dinv64, dinv32, st);
  return o.kind == RB_PROP_NODE
             ? launch_femlhs<false, RB_PROP_NODE>(m, o, evol, ddd, dco, val64, val32, dinv64, dinv32, st)
             : launch_femlhs<false, RB_PROP_ELEM>(m, o, evol, ddd, dco, val64, val32, dinv64, dinv32, st);
}

// --------------------------------------------------------------------------
// Assembly for callers that cannot allocate device memory.
//
// rb_femlhs needs one scratch array (the diffusion coefficient per node or
// per tet) and takes it from a caller-provided workspace.  Some callers have
// no way to provide one: host code in another language that binds this C ABI
// and owns only its own input/output buffers, or code that runs where a
// cudaMalloc is not allowed (it would synchronise the device, or the memory
// pool belongs to someone else).  rb_femlhs_noalloc gives them the same
// assembly with the scratch taken from a fixed array compiled into this
// library instead.
namespace rb {

// Capacity of the fixed scratch: 4,194,304 doubles (32 MiB), i.e. meshes with
// up to that many nodes (per-node properties) or tets (per-tet properties).
// Every GPU that loads this library keeps these 32 MiB until the process ends.
constexpr int64_t kNoallocScratchMax = 4 * 1024 * 1024;
static __device__ __align__(256) double g_noalloc_dco[kNoallocScratchMax];

// Host code cannot use g_noalloc_dco directly (on the host that name is only a
// stand-in for the device array); its device address is looked up once per
// device, with that device current, and cached here.
constexpr int kNoallocMaxDevices = 64;
static std::mutex g_noalloc_mu;
static double* g_noalloc_ptr[kNoallocMaxDevices] = {};

static int noalloc_scratch(double** out) {
  int dev = -1;
  RB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoallocMaxDevices)
    return fail(RB_EARG, "rb_femlhs_noalloc: device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_dco);
    if (e != cudaSuccess || !p)
      return fail(RB_ECUDA, "rb_femlhs_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev,
                  cudaGetErrorString(e));
    g_noalloc_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return RB_OK;
}

}  // namespace rb

extern "C" int rb_femlhs_noalloc(const rb_mesh* mesh, const rb_optics* optics, const double* evol,
                                 const double* ddd, void* val64, void* val32, void* dinv64, void* dinv32,
                                 void* stream) {
  if (!mesh || !optics || !val64 || !evol || !ddd)
    return fail(RB_EARG, "rb_femlhs_noalloc: mesh, optics, evol, ddd and val64 are required");
  const rb_mesh& m = *mesh;
  const rb_optics& o = *optics;
  if (o.kind != RB_PROP_NODE && o.kind != RB_PROP_ELEM) return fail(RB_EARG, "rb_femlhs_noalloc: bad property kind");
  const int64_t np = (o.kind == RB_PROP_NODE) ? m.nn : m.ne;
  if (m.nn < 1 || np < 1)
    return fail(RB_EARG, "rb_femlhs_noalloc: empty mesh (%lld nodes, %lld tets)", (long long)m.nn, (long long)m.ne);
  if (np > kNoallocScratchMax)
    return fail(RB_ESIZE,
                "rb_femlhs_noalloc: %lld %s exceed the fixed scratch of %lld entries; use rb_femlhs with a workspace",
                (long long)np, o.kind == RB_PROP_NODE ? "nodes" : "tets", (long long)kNoallocScratchMax);
  if (!m.elem || !m.indptr || !m.indices || !m.node_eptr || !m.node_elist || !m.node_fptr)
    return fail(RB_EARG, "rb_femlhs_noalloc: mesh arrays missing");
  if (m.nf > 0 && (!m.face || !m.area || !m.node_flist))
    return fail(RB_EARG, "rb_femlhs_noalloc: boundary arrays missing");
  if (!o.mua || !o.musp) return fail(RB_EARG, "rb_femlhs_noalloc: mua and musp are required");
  if (!(o.omega >= 0.0)) return fail(RB_EARG, "rb_femlhs_noalloc: omega must be >= 0");
  double* dco = nullptr;
  RB_TRY(noalloc_scratch(&dco));
  // the prologue kernel overwrites every scratch entry the assembly reads, so
  // nothing left by an earlier call needs clearing
  cudaStream_t st = as_stream(stream);
  if (o.omega > 0.0)
    return o.kind == RB_PROP_NODE
               ? launch_femlhs<true, RB_PROP_NODE>(m, o, evol, ddd, dco, val64, val32, dinv64, dinv32, st)
               : launch_femlhs<true, RB_PROP_ELEM>(m, o, evol, ddd, dco, val64, val32, dinv64, dinv32, st);
  return o.kind == RB_PROP_NODE
             ? launch_femlhs<false, RB_PROP_NODE>(m, o, evol, ddd, dco, val64, val32, dinv64, dinv32, st)
             : launch_femlhs<false, RB_PROP_ELEM>(m, o, evol, ddd, dco, val64, val32, dinv64, dinv32, st);
}

namespace rb {
// label table -> per-tet mua, musp (seg clipped like np.clip(seg, 0, nlabel - 1))
__global__ void prop_labels_kernel(const int32_t* __restrict__ seg, int64_t ne, const double* __restrict__ tab,
                                   int64_t nlabel, int ncol, double* __restrict__ mua, double* __restrict__ musp) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne; e += (int64_t)gridDim.x * blockDim.x) {
    int64_t l = seg[e];
    l = l < 0 ? 0 : (l >= nlabel ? nlabel - 1 : l);
    const double* t = tab + l * ncol;
    mua[e] = t[0];
    musp[e] = ncol >= 3 ? t[1] * (1.0 - t[2]) : t[1];
  }
}
}  // namespace rb

extern "C" int rb_prop_from_labels(const int32_t* seg, int64_t ne, const double* tab, int64_t nlabel, int32_t ncol,
                                   double* mua_out, double* musp_out, void* stream) {
  if (!seg || !tab || !mua_out || !musp_out || ne < 0 || nlabel < 1 || ncol < 2)
    return fail(RB_EARG, "rb_prop_from_labels: bad arguments");
  if (ne == 0) return RB_OK;
  prop_labels_kernel<<<(unsigned)std::min<int64_t>(ceil_div(ne, 256), 148 * 16), 256, 0, as_stream(stream)>>>(
      seg, ne, tab, nlabel, ncol, mua_out, musp_out);
  RB_LAUNCH_CHECK();
  return RB_OK;
}
