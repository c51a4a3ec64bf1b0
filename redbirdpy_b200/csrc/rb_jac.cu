// Adjoint Jacobians written straight into node rows.
//
// For every source/detector pair k and node n the Jacobian entry is a
// bilinear form over the nodes N(n) that share a tet with n (the CSR row of
// n):  J[k][n] = sum_{a,b in N(n)} phi_s(k)[a] B_n[a][b] phi_d(k)[b],  with
// B_n = sum over tets e containing n of a 4x4 coefficient block w_e:
//   mua, reference semantics:  w_e(i,j) = -0.025 V_e (1 + d_ij) / 2
//        (element mass 0.1 V (diag + cross/2) then 1/4 lumping, forward.py:509-569)
//   mua, node-based exact:     w_e(i,j) = -V_e/120 (1 + d_ni + d_nj)(1 + d_ij)
//   D (diffusion), exact:      w_e(i,j) = -1/4 V_e grad(l_i).grad(l_j)
// A CTA takes TN consecutive nodes: it stages the phi rows of their
// neighbours for every column the pairs use, builds the TN small B_n, forms
// C_n = B_n Phi_det once per detector, and then every pair costs |N(n)|
// multiply-adds: J[k][n] = sum_a phi_s(k)[a] C_n[a][d(k)].  Threads that
// write one row segment are consecutive, so the nsd x nn output (the
// dominant HBM traffic) is written in full sectors.
#include <cuda_bf16.h>

#include <algorithm>
#include <type_traits>

#include "rb_common.cuh"
#include "rb_tc.cuh"

namespace rb {

enum { JAC_MUA_REF = 0, JAC_MUA_NODAL = 1, JAC_D = 2 };
constexpr int kJacThreads = 256;

template <typename C> struct JacT;
template <> struct JacT<float> { typedef float real; };
template <> struct JacT<double> { typedef double real; };
template <> struct JacT<cfloat> { typedef float real; };
template <> struct JacT<cdouble> { typedef double real; };

template <typename C, typename In> __device__ __forceinline__ C cvt(In v);
template <> __device__ __forceinline__ float cvt<float, float>(float v) { return v; }
template <> __device__ __forceinline__ float cvt<float, double>(double v) { return (float)v; }
template <> __device__ __forceinline__ double cvt<double, float>(float v) { return v; }
template <> __device__ __forceinline__ double cvt<double, double>(double v) { return v; }
template <> __device__ __forceinline__ cfloat cvt<cfloat, cfloat>(cfloat v) { return v; }
template <> __device__ __forceinline__ cfloat cvt<cfloat, cdouble>(cdouble v) { return make_float2((float)v.x, (float)v.y); }
template <> __device__ __forceinline__ cdouble cvt<cdouble, cfloat>(cfloat v) { return make_double2(v.x, v.y); }
template <> __device__ __forceinline__ cdouble cvt<cdouble, cdouble>(cdouble v) { return v; }

__device__ __forceinline__ float scale_r(float b, float v) { return b * v; }
__device__ __forceinline__ double scale_r(double b, double v) { return b * v; }
__device__ __forceinline__ cfloat scale_r(float b, cfloat v) { return make_float2(b * v.x, b * v.y); }
__device__ __forceinline__ cdouble scale_r(double b, cdouble v) { return make_double2(b * v.x, b * v.y); }

__device__ __forceinline__ int tid_warp() { return (int)(threadIdx.x >> 5); }

struct JacArgs {
  const int32_t* indptr;
  const int32_t* indices;
  const int32_t* eptr;
  const int32_t* elist;
  const int32_t* elem;
  const double* evol;   // ne tet volumes
  const double* ddd;    // ne x 10 deldotdel (RB_JAC_D only)
  int64_t nn;
  const int32_t* cols;  // nc staged phi columns
  int32_t nc, det0, ndet;
  const int32_t* psrc;  // nsd: staged slot of the source column
  const int32_t* pdet;  // nsd: 0..ndet-1 index of the detector
  int64_t nsd, ld, ldj;
  int32_t rmax, emax, what;
  int32_t grid;  // pairs are all (source slot, detector) combinations, detector-major
  int64_t node0;  // first node of the range (J column 0); nn is the range's end
};

// Per-node strides of the staged phi and C blocks, padded so that the TN
// nodes a warp covers land in different shared-memory banks: with E
// elements per 128-byte bank row, the phi stride is 1 (mod E) and the C
// stride E/4 (mod E).
template <typename C> __host__ __device__ inline int jac_phi_stride(int rmax, int nc) {
  constexpr int E = 128 / (int)sizeof(C);
  return (rmax * nc + E - 1) / E * E + 1;
}
template <typename C> __host__ __device__ inline int jac_c_stride(int rmax, int nd) {
  constexpr int E = 128 / (int)sizeof(C);
  return (rmax * nd + E - 1) / E * E + E / 4;
}

// smem layout, TN nodes, each region starting on a 16-byte boundary:
//   phi [TN][phi stride] C | Bm [TN][rmax][rmax] R | Cm [TN][C stride] C |
//   W [TN][emax][16] R | EN [TN][emax] int4 | nb [TN][rmax] int | rn, ek [TN] int |
//   LP [TN][emax][4] int16 (position of each tet node in the node's row)
__host__ __device__ inline size_t al16(size_t b) { return (b + 15) / 16 * 16; }
struct JacSmem {
  size_t phi, B, C, W, EN, nb, lp, total;
};
template <typename C>
__host__ __device__ inline JacSmem jac_layout(int TN, int rmax, int nc, int ndet, int emax) {
  typedef typename JacT<C>::real R;
  JacSmem L;
  L.phi = 0;
  L.B = L.phi + al16((size_t)TN * jac_phi_stride<C>(rmax, nc) * sizeof(C));
  L.C = L.B + al16((size_t)TN * rmax * rmax * sizeof(R));
  L.W = L.C + al16((size_t)TN * jac_c_stride<C>(rmax, ndet) * sizeof(C));
  L.EN = L.W + al16((size_t)TN * emax * 16 * sizeof(R));
  L.nb = L.EN + al16((size_t)TN * emax * sizeof(int4));
  L.lp = L.nb + al16((size_t)TN * rmax * sizeof(int) + TN * sizeof(int) * 2);
  L.total = L.lp + al16((size_t)TN * emax * 4 * sizeof(int16_t));
  return L;
}
template <typename C>
__host__ __device__ inline size_t jac_smem(int TN, int rmax, int nc, int ndet, int emax) {
  return jac_layout<C>(TN, rmax, nc, ndet, emax).total;
}

// one Jacobian entry: complex values split into a real-part and an
// imaginary-part row block (SPLIT), optionally rounded to BF16 (BF)
template <typename C, bool SPLIT, bool BF, bool NARROW = false>
__device__ __forceinline__ void jac_store(void* Jout, int64_t nsd, int64_t ldj, int64_t k, int64_t n, C v) {
  typedef typename JacT<C>::real R;
  if constexpr (NARROW) {  // computed in FP64, stored as FP32 rows
    float* Jf = reinterpret_cast<float*>(Jout);
    if constexpr (SPLIT) {
      Jf[k * ldj + n] = (float)v.x;
      Jf[(nsd + k) * ldj + n] = (float)v.y;
    } else {
      Jf[k * ldj + n] = (float)v;
    }
  } else if constexpr (SPLIT) {
    if constexpr (BF) {
      __nv_bfloat16* Jb = reinterpret_cast<__nv_bfloat16*>(Jout);
      Jb[k * ldj + n] = __float2bfloat16_rn(v.x);
      Jb[(nsd + k) * ldj + n] = __float2bfloat16_rn(v.y);
    } else {
      R* Jr = reinterpret_cast<R*>(Jout);
      Jr[k * ldj + n] = v.x;
      Jr[(nsd + k) * ldj + n] = v.y;
    }
  } else if constexpr (BF) {
    reinterpret_cast<__nv_bfloat16*>(Jout)[k * ldj + n] = __float2bfloat16_rn(v);
  } else {
    reinterpret_cast<C*>(Jout)[k * ldj + n] = v;
  }
}

// Steps 1-3 of a CTA's TN nodes (n0 ..): stage the neighbours' phi rows
// (every column the pairs use, converted to C), build each node's B_n and
// C_n = B_n Phi_det in shared memory (layout jac_layout).  Ends with a
// barrier; step 4 (the pair products) is the caller's.
template <typename C, typename In, int TN>
__device__ __forceinline__ void jac_stage(const JacArgs& a, const In* __restrict__ phi, unsigned char* smem,
                                          int64_t n0) {
  typedef typename JacT<C>::real R;
  const int rmax = a.rmax, nc = a.nc, nd = a.ndet, emax = a.emax;
  const int SP = jac_phi_stride<C>(rmax, nc), SC = jac_c_stride<C>(rmax, nd);
  const JacSmem L = jac_layout<C>(TN, rmax, nc, nd, emax);
  C* sphi = reinterpret_cast<C*>(smem + L.phi);
  R* sB = reinterpret_cast<R*>(smem + L.B);
  C* sC = reinterpret_cast<C*>(smem + L.C);
  R* sW = reinterpret_cast<R*>(smem + L.W);
  int4* sEN = reinterpret_cast<int4*>(smem + L.EN);
  int* snb = reinterpret_cast<int*>(smem + L.nb);
  int* srn = snb + TN * rmax;
  int* sek = srn + TN;
  int16_t* slp = reinterpret_cast<int16_t*>(smem + L.lp);
  const int warp = tid_warp(), lane = threadIdx.x & 31;
  constexpr int kWarps = kJacThreads / 32;
  const int tid = threadIdx.x;
  // 1. rows and incident tets of the TN nodes
  if (tid < TN) {
    const int64_t n = n0 + tid;
    srn[tid] = (n < a.nn) ? a.indptr[n + 1] - a.indptr[n] : 0;
    sek[tid] = (n < a.nn) ? a.eptr[n + 1] - a.eptr[n] : 0;
  }
  __syncthreads();
  for (int i = tid; i < TN * rmax; i += kJacThreads) {
    const int t = i / rmax, q = i % rmax;
    snb[i] = (q < srn[t]) ? a.indices[a.indptr[n0 + t] + q] : -1;
  }
  // per (node, incident tet): node ids and the 16 coefficients w_e(i,j)
  for (int i = tid; i < TN * emax; i += kJacThreads) {
    const int t = i / emax, q = i % emax;
    if (q >= sek[t]) continue;
    const int64_t n = n0 + t;
    const int32_t e = a.elist[a.eptr[n] + q];
    const int4 en = reinterpret_cast<const int4*>(a.elem)[e];
    sEN[i] = en;
    const int32_t nd4[4] = {en.x, en.y, en.z, en.w};
    const double vol = a.evol[e];
    const double* dd = a.ddd ? a.ddd + 10 * (int64_t)e : nullptr;
    R* W = sW + (size_t)i * 16;
    for (int ii = 0; ii < 4; ++ii)
      for (int jj = 0; jj < 4; ++jj) {
        double wv;
        if (a.what == JAC_MUA_REF) {
          wv = -0.0125 * vol * (ii == jj ? 2.0 : 1.0);
        } else if (a.what == JAC_MUA_NODAL) {
          const double f = 1.0 + (nd4[ii] == n) + (nd4[jj] == n);
          wv = -vol / 120.0 * f * (ii == jj ? 2.0 : 1.0);
        } else {
          // upper-triangle index of (min, max) in the 10-entry deldotdel row
          const int lo = ii < jj ? ii : jj, hi = ii < jj ? jj : ii;
          wv = -0.25 * dd[lo * 4 - lo * (lo - 1) / 2 + (hi - lo)];
        }
        W[ii * 4 + jj] = (R)wv;
      }
  }
  __syncthreads();
  // staged phi rows of the neighbours, converted to the compute type: a warp
  // per (node, neighbour) slot, lanes over the columns
  for (int slot = warp; slot < TN * rmax; slot += kWarps) {
    const int t = slot / rmax, q = slot - t * rmax;
    const int nb = snb[slot];
    C* dst = sphi + (size_t)t * SP + (size_t)q * nc;
    for (int c = lane; c < nc; c += 32) dst[c] = nb >= 0 ? cvt<C, In>(phi[(int64_t)nb * a.ld + a.cols[c]]) : s_zero(C());
  }
  // position of each tet node in its node's row (every tet node is a neighbour)
  for (int i = tid; i < TN * emax * 4; i += kJacThreads) {
    const int tq = i >> 2, m = i & 3;
    const int t = tq / emax, q = tq - t * emax;
    int pos = -1;
    if (q < sek[t]) {
      const int4 en = sEN[tq];
      const int node = m == 0 ? en.x : m == 1 ? en.y : m == 2 ? en.z : en.w;
      for (int b = 0; b < srn[t]; ++b)
        if (snb[t * rmax + b] == node) pos = b;
    }
    slp[i] = (int16_t)pos;
  }
  __syncthreads();
  // 2. B_n[a][b] = sum over the node's tets (ascending) of w_e at the local
  // positions: a thread per row a walks the tets holding it and adds its 4
  // coefficients into the row (per entry the same order as summing over the
  // tets for each (a, b) separately)
  for (int row = tid; row < TN * rmax; row += kJacThreads) {
    const int t = row / rmax, ia = row - t * rmax;
    R* Brow = sB + (size_t)row * rmax;
    for (int ib = 0; ib < rmax; ++ib) Brow[ib] = 0;
    if (ia < srn[t]) {
      for (int q = 0; q < sek[t]; ++q) {
        const int16_t* lp = slp + ((size_t)t * emax + q) * 4;
        int pa = -1;
#pragma unroll
        for (int m = 0; m < 4; ++m)
          if (lp[m] == ia) pa = m;
        if (pa < 0) continue;
        const R* W = sW + ((size_t)t * emax + q) * 16 + pa * 4;
#pragma unroll
        for (int m = 0; m < 4; ++m)
          if (lp[m] >= 0) Brow[lp[m]] += W[m];  // (a tet node outside the row would be a broken pattern)
      }
    }
  }
  __syncthreads();
  // 3. C_n[a][d] = sum_b B_n[a][b] phi[b][det d]: a warp per (node, row a),
  // lanes over the detectors
  for (int slot = warp; slot < TN * rmax; slot += kWarps) {
    const int t = slot / rmax, ia = slot - t * rmax;
    const int nr = srn[t];
    const R* Brow = sB + (size_t)slot * rmax;
    const C* P = sphi + (size_t)t * SP + a.det0;
    C* Cout = sC + (size_t)t * SC + (size_t)ia * nd;
    for (int d = lane; d < nd; d += 32) {
      C s = s_zero(C());
      if (ia < nr)
        for (int b = 0; b < nr; ++b) s = s_add(s, scale_r(Brow[b], P[(size_t)b * nc + d]));
      Cout[d] = s;
    }
  }
  __syncthreads();
}

template <typename C, typename In, int TN, bool SPLIT, bool GRID, bool BF, bool NARROW = false>
__global__ void __launch_bounds__(kJacThreads)
jac_kernel(JacArgs a, const In* __restrict__ phi, void* __restrict__ Jout) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int rmax = a.rmax, nc = a.nc, nd = a.ndet, emax = a.emax;
  const int SP = jac_phi_stride<C>(rmax, nc), SC = jac_c_stride<C>(rmax, nd);
  const JacSmem L = jac_layout<C>(TN, rmax, nc, nd, emax);
  const C* sphi = reinterpret_cast<const C*>(smem + L.phi);
  const C* sC = reinterpret_cast<const C*>(smem + L.C);
  const int* srn = reinterpret_cast<const int*>(smem + L.nb) + TN * rmax;

  const int64_t n0 = a.node0 + (int64_t)blockIdx.x * TN;
  const int tid = threadIdx.x;
  jac_stage<C, In, TN>(a, phi, smem, n0);
  // 4. J[k][n] = sum_a phi[a][src k] C_n[a][det k]
  if constexpr (GRID) {
    // all (source, detector) combinations, k = d * nsrc + s (sdmap's
    // detector-major order): a thread takes 4 sources x 4 detectors of one
    // node, so each staged value read from shared memory feeds 4 products
    const int nsu = a.det0, nsb = nsu / 4, ndb = nd / 4;
    const int items = nsb * ndb * TN;
    for (int i = tid; i < items; i += kJacThreads) {
      const int t = i % TN, pb = i / TN;
      const int sb = pb % nsb, db = pb / nsb;
      const int64_t n = n0 + t;
      if (n >= a.nn) continue;
      C acc[4][4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = s_zero(C());
      for (int ia = 0; ia < srn[t]; ++ia) {
        const C* P = sphi + (size_t)t * SP + (size_t)ia * nc + sb * 4;
        const C* Cn = sC + (size_t)t * SC + (size_t)ia * nd + db * 4;
        C pv[4], cv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          pv[u] = P[u];
          cv[u] = Cn[u];
        }
        if constexpr (std::is_same<C, cfloat>::value) {
          // packed FP32x2 FMAs, two per complex product, in s_fma's order:
          // (x, y) += (-a.y, a.y) (b.y, b.x), then += (a.x, a.x) (b.x, b.y)
          float2 ayy[4], axx[4], bsw[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            ayy[u] = make_float2(-pv[u].y, pv[u].y);
            axx[u] = make_float2(pv[u].x, pv[u].x);
            bsw[u] = make_float2(cv[u].y, cv[u].x);
          }
#pragma unroll
          for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[u][v] = __ffma2_rn(axx[u], cv[v], __ffma2_rn(ayy[u], bsw[v], acc[u][v]));
        } else {
#pragma unroll
          for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[u][v] = s_fma(pv[u], cv[v], acc[u][v]);
        }
      }
#pragma unroll
      for (int v = 0; v < 4; ++v)
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int64_t k = (int64_t)(db * 4 + v) * nsu + sb * 4 + u;
          jac_store<C, SPLIT, BF, NARROW>(Jout, a.nsd, a.ldj, k, n - a.node0, acc[u][v]);
        }
    }
    return;
  }
  // general pair list: t fastest -> row segments
  const int64_t total = a.nsd * TN;
  for (int64_t i = tid; i < total; i += kJacThreads) {
    const int t = (int)(i % TN);
    const int64_t k = i / TN;
    const int64_t n = n0 + t;
    if (n >= a.nn) continue;
    const int ps = a.psrc[k], pd = a.pdet[k];
    const C* P = sphi + (size_t)t * SP + ps;
    const C* Cn = sC + (size_t)t * SC + pd;
    C s = s_zero(C());
    for (int ia = 0; ia < srn[t]; ++ia) s = s_fma(P[(size_t)ia * nc], Cn[(size_t)ia * nd], s);
    // complex rows are split into a block of real parts and a block of
    // imaginary parts (matreform 'real', recon.py:532-546)
    jac_store<C, SPLIT, BF, NARROW>(Jout, a.nsd, a.ldj, k, n - a.node0, s);
  }
}

// Element Jacobian, reference semantics (forward.py:509-558):
// Je[k][e] = -0.1 V (sum_i ps_i pd_i + 1/2 sum_{i!=j} ps_i pd_j)
template <typename T>
__global__ void jac_elem_kernel(const double* __restrict__ evol, const int32_t* __restrict__ elem, int64_t ne,
                                const T* __restrict__ phi, int64_t ld, const int32_t* __restrict__ scol,
                                const int32_t* __restrict__ dcol, int64_t nsd, T* __restrict__ Je) {
  const int64_t total = nsd * ne;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = i / ne, e = i % ne;
    const int4 en = reinterpret_cast<const int4*>(elem)[e];
    const int32_t nd4[4] = {en.x, en.y, en.z, en.w};
    const double vol = evol[e];
    const int s = scol[k], d = dcol[k];
    T ss = s_zero(T()), sd = s_zero(T()), dg = s_zero(T());
    for (int m = 0; m < 4; ++m) {
      const T a = phi[(int64_t)nd4[m] * ld + s], b = phi[(int64_t)nd4[m] * ld + d];
      ss = s_add(ss, a);
      sd = s_add(sd, b);
      dg = s_fma(a, b, dg);
    }
    // diag + (total - diag)/2 = (diag + ss*sd)/2
    const T tot = s_fma(ss, sd, dg);
    Je[i] = scale_r((typename JacT<T>::real)(-0.05 * vol), tot);
  }
}

// ------------------------------------------- step 4 on the tensor cores
// For the full (source x detector) grid with FP32 output, the pair products
// of node t, P_t[s][d] = sum_a phi[a][s] C_t[a][d], are one tcgen05 MMA
// D_t (128 x N) = A_t (128 x K) B_t^T (N x K), K along the node's row:
//   B_t row n = source n: Re phi[a][n] for a < k8, then Im phi[a][n];
//   A_t row d (d < ndet): Re C[a][d], then -Im C[a][d];
//   A_t row 64 + d (complex): Im C[a][d], then Re C[a][d];
// so that D row d holds Re P[.][d] and D row 64 + d Im P[.][d] (real
// fields: K = k8, rows d only).  k8 = rmax rounded up to 8.  The operands
// are written into shared memory in the 128-byte-swizzled K-major layout
// (rb_tc.cuh) as TF32 pairs x = hi + lo, and D = hi hi + hi lo + lo hi
// (three MMAs per 8-wide K step) keeps FP32 accuracy.  The TN accumulators
// (N columns each) stay in tensor memory until the epilogue: a thread owns
// one D row (one detector, real or imaginary part) and writes, per source,
// the TN consecutive node columns of that J row at once.
constexpr int kJtcTN = 4;

struct JtcLayout {
  size_t ahi, alo, bhi, blo, bar, total;
  int Kp, N, k8;
};

template <typename C>
__host__ __device__ inline JtcLayout jtc_layout(int rmax, int nc, int ndet, int emax, int nsu) {
  JtcLayout T;
  T.k8 = (rmax + 7) / 8 * 8;
  T.Kp = Scalar<C>::is_complex ? 2 * T.k8 : T.k8;
  T.N = (nsu + 31) / 32 * 32;
  size_t o = (jac_smem<C>(kJtcTN, rmax, nc, ndet, emax) + 1023) / 1024 * 1024;
  // a swizzle atom row is 128 bytes (32 TF32) whatever Kp: whole atoms
  const int atoms = (T.Kp + 31) / 32;
  const size_t ab = (size_t)128 * 128 * atoms, bb = (size_t)T.N * 128 * atoms;  // multiples of 1024
  T.ahi = o;
  T.alo = o + ab;
  T.bhi = o + 2 * ab;
  T.blo = o + 2 * ab + bb;
  T.bar = o + 2 * ab + 2 * bb;
  T.total = T.bar + 64 + 1024;  // the kernel aligns its base up to 1024 bytes
  return T;
}

// byte offset of element (r, k) of a K-major 128-byte-swizzled operand of R
// rows: K atoms of 32 elements are R x 128-byte blocks one after the other
__device__ __forceinline__ uint32_t sw128_off(int r, int k, int R) {
  const int atom = k >> 5, kk = k & 31;
  return (uint32_t)(atom * R * 128 + (r >> 3) * 1024 + (r & 7) * 128 + (((kk >> 2) ^ (r & 7)) << 4) + ((kk & 3) << 2));
}

__device__ __forceinline__ void tf32_split(float x, float& hi, float& lo) {
  uint32_t h, l;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
  hi = __uint_as_float(h);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(x - hi));
  lo = __uint_as_float(l);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}

template <typename C, typename In>
__global__ void __launch_bounds__(kJacThreads, 1)
jac_tc_kernel(JacArgs a, const In* __restrict__ phi, float* __restrict__ Jout, uint32_t tmem_cols,
              int* __restrict__ err) {
  constexpr bool CPLX = Scalar<C>::is_complex;
  constexpr int TN = kJtcTN;
  extern __shared__ __align__(1024) unsigned char jsm_raw[];
  unsigned char* smem =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(jsm_raw) + 1023) & ~uintptr_t(1023));
  const int rmax = a.rmax, nc = a.nc, nd = a.ndet, emax = a.emax, nsu = a.det0;
  const JtcLayout T = jtc_layout<C>(rmax, nc, nd, emax, nsu);
  const JacSmem L = jac_layout<C>(TN, rmax, nc, nd, emax);
  const int SP = jac_phi_stride<C>(rmax, nc), SC = jac_c_stride<C>(rmax, nd);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + T.bar);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
  int* sflag = reinterpret_cast<int*>(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    mbar_init(smem_u32(bar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *sflag = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  const int64_t n0 = a.node0 + (int64_t)blockIdx.x * TN;
  jac_stage<C, In, TN>(a, phi, smem, n0);
  const C* sphi = reinterpret_cast<const C*>(smem + L.phi);
  const C* sC = reinterpret_cast<const C*>(smem + L.C);
  const int* srn = reinterpret_cast<const int*>(smem + L.nb) + TN * rmax;
  const int Kp = T.Kp, N = T.N, k8 = T.k8;
  unsigned char* Ahi = smem + T.ahi;
  unsigned char* Alo = smem + T.alo;
  unsigned char* Bhi = smem + T.bhi;
  unsigned char* Blo = smem + T.blo;
  const uint32_t idesc = umma_idesc(2, 128, (uint32_t)N);
  int nmma = 0;  // commits issued (parity of the next wait)
  bool ok = true;
  for (int t = 0; t < TN && ok; ++t) {
    const int rn = srn[t];
    // consecutive threads take consecutive rows of one K column: the staged
    // C and phi values they read are consecutive in shared memory
    for (int i = tid; i < 128 * Kp; i += kJacThreads) {
      const int k = i >> 7, m = i & 127;
      float x = 0.f;
      if constexpr (CPLX) {
        const int hk = k >= k8 ? 1 : 0, q = k - hk * k8;
        const int d = m < 64 ? m : m - 64;
        if (q < rn && d < nd) {
          const C c = sC[(size_t)t * SC + (size_t)q * nd + d];
          x = (m < 64) ? (hk ? -c.y : c.x) : (hk ? c.x : c.y);
        }
      } else {
        if (k < rn && m < nd) x = sC[(size_t)t * SC + (size_t)k * nd + m];
      }
      float h, l;
      tf32_split(x, h, l);
      const uint32_t off = sw128_off(m, k, 128);
      *reinterpret_cast<float*>(Ahi + off) = h;
      *reinterpret_cast<float*>(Alo + off) = l;
    }
    for (int i = tid; i < N * Kp; i += kJacThreads) {
      const int k = i / N, n = i - k * N;
      float x = 0.f;
      if constexpr (CPLX) {
        const int hk = k >= k8 ? 1 : 0, q = k - hk * k8;
        if (q < rn && n < nsu) {
          const C v = sphi[(size_t)t * SP + (size_t)q * nc + n];
          x = hk ? v.y : v.x;
        }
      } else {
        if (k < rn && n < nsu) x = sphi[(size_t)t * SP + (size_t)k * nc + n];
      }
      float h, l;
      tf32_split(x, h, l);
      const uint32_t off = sw128_off(n, k, N);
      *reinterpret_cast<float*>(Bhi + off) = h;
      *reinterpret_cast<float*>(Blo + off) = l;
    }
    // the operands written by the threads become visible to the tensor cores
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t dcol = tmem + (uint32_t)(t * N);
      const uint32_t ah = smem_u32(Ahi), al = smem_u32(Alo), bh = smem_u32(Bhi), bl = smem_u32(Blo);
      for (int j = 0; j < Kp / 8; ++j) {
        const uint32_t ao = (uint32_t)((j >> 2) * 128 * 128 + (j & 3) * 32);
        const uint32_t bo = (uint32_t)((j >> 2) * N * 128 + (j & 3) * 32);
        umma_tf32_i(dcol, umma_desc_sw128(ah + ao), umma_desc_sw128(bh + bo), idesc, j > 0 ? 1u : 0u);
        umma_tf32_i(dcol, umma_desc_sw128(ah + ao), umma_desc_sw128(bl + bo), idesc, 1u);
        umma_tf32_i(dcol, umma_desc_sw128(al + ao), umma_desc_sw128(bh + bo), idesc, 1u);
      }
      umma_commit(smem_u32(bar));
      // the next node's operands overwrite these: wait for the MMAs to read them
      if (!mbar_wait(smem_u32(bar), (uint32_t)(nmma & 1), err, 1)) *sflag = 1;
    }
    ++nmma;
    __syncthreads();
    if (*sflag) ok = false;
  }
  if (ok) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // warp w reads tensor-memory lanes 32 (w % 4) ..: D row m; warps 0-3
    // take the first half of the sources, warps 4-7 the second
    const int q = warp & 3, m = 32 * q + lane, hf = warp >> 2;
    int d = -1;
    bool im = false;
    if (m < nd) {
      d = m;
    } else if (CPLX && m >= 64 && m - 64 < nd) {
      d = m - 64;
      im = true;
    }
    const int64_t c0 = n0 - a.node0;  // J column of the CTA's first node
    const int nval = (int)((a.nn - n0) < TN ? (a.nn - n0) : TN);
    for (int s0 = hf * (N / 2); s0 < (hf + 1) * (N / 2); s0 += 16) {
      uint32_t v[TN][16];
#pragma unroll
      for (int t = 0; t < TN; ++t) tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(t * N + s0), v[t]);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (d >= 0) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
          const int sidx = s0 + u;
          if (sidx >= nsu) break;
          const int64_t row = (im ? a.nsd : 0) + (int64_t)d * nsu + sidx;
          float* dst = Jout + row * a.ldj + c0;
          if (nval == TN && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
            *reinterpret_cast<float4*>(dst) = make_float4(__uint_as_float(v[0][u]), __uint_as_float(v[1][u]),
                                                          __uint_as_float(v[2][u]), __uint_as_float(v[3][u]));
          } else {
#pragma unroll
            for (int t = 0; t < TN; ++t)
              if (t < nval) dst[t] = __uint_as_float(v[t][u]);
          }
        }
      }
    }
  } else if (tid == 0) {
    // a wait gave up: let the MMAs in flight finish before the memory goes
    mbar_wait(smem_u32(bar), (uint32_t)((nmma - 1) & 1), err, 2);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols));
}

// the tensor-core path: its error word (a bounded wait that gave up) and the
// switch that lets a caller take the SIMT products instead
__device__ int g_jac_tc_err;
static bool g_jac_tc_on = false;

// launches the tensor-core form when the pairs are the full grid with FP32
// output and the sizes fit it; returns 1 when it did not apply
template <typename C, typename In>
static int launch_jac_tc(const JacArgs& a, const void* phi, void* J, cudaStream_t st, int* launched) {
  *launched = 0;
  if (!g_jac_tc_on || !a.grid) return RB_OK;
  const int nsu = a.det0;
  if (a.rmax > 32 || nsu < 1 || nsu > 128 || a.ndet > (Scalar<C>::is_complex ? 64 : 128)) return RB_OK;
  const JtcLayout T = jtc_layout<C>(a.rmax, a.nc, a.ndet, a.emax, nsu);
  if (T.total > 220 * 1024) return RB_OK;
  uint32_t cols = 32;
  while (cols < (uint32_t)(kJtcTN * T.N)) cols <<= 1;
  if (cols > 512) return RB_OK;
  int* err = nullptr;
  RB_CUDA_TRY(cudaGetSymbolAddress(reinterpret_cast<void**>(&err), g_jac_tc_err));
  RB_CUDA_TRY(cudaFuncSetAttribute(jac_tc_kernel<C, In>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T.total));
  const unsigned g = (unsigned)ceil_div(a.nn - a.node0, kJtcTN);
  jac_tc_kernel<C, In><<<g, kJacThreads, T.total, st>>>(a, (const In*)phi, (float*)J, cols, err);
  RB_LAUNCH_CHECK();
  *launched = 1;
  return RB_OK;
}

template <typename C, typename In, bool SPLIT, bool GRID, bool BF, bool NARROW = false>
static int launch_jac_t(const JacArgs& a, const void* phi, void* J, cudaStream_t st) {
  int TN = 8;
  const size_t budget = 110 * 1024;
  while (TN > 1 && jac_smem<C>(TN, a.rmax, a.nc, a.ndet, a.emax) > budget) TN >>= 1;
  const size_t sm = jac_smem<C>(TN, a.rmax, a.nc, a.ndet, a.emax);
  if (sm > 200 * 1024) return fail(RB_ESIZE, "rb_jac: staging needs %zu bytes of shared memory", sm);
  const unsigned g = (unsigned)ceil_div(a.nn - a.node0, TN);
#define RB_JL(TN_)                                                                                     \
  do {                                                                                                 \
    RB_CUDA_TRY(cudaFuncSetAttribute(jac_kernel<C, In, TN_, SPLIT, GRID, BF, NARROW>,                  \
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));           \
    jac_kernel<C, In, TN_, SPLIT, GRID, BF, NARROW><<<g, kJacThreads, sm, st>>>(a, (const In*)phi, J);   \
  } while (0)
  switch (TN) {
    case 8: RB_JL(8); break;
    case 4: RB_JL(4); break;
    case 2: RB_JL(2); break;
    default: RB_JL(1); break;
  }
#undef RB_JL
  RB_LAUNCH_CHECK();
  return RB_OK;
}

template <typename C, typename In, bool SPLIT = false, bool BF = false, bool NARROW = false>
static int launch_jac(const JacArgs& a, const void* phi, void* J, cudaStream_t st) {
  // FP32 rows (complex ones split into real and imaginary blocks): the pair
  // products on the tensor cores when the sizes allow
  if constexpr (!BF && !NARROW && ((std::is_same<C, cfloat>::value && SPLIT) || std::is_same<C, float>::value)) {
    int done = 0;
    RB_TRY((launch_jac_tc<C, In>(a, phi, J, st, &done)));
    if (done) return RB_OK;
  }
  if (a.grid) return launch_jac_t<C, In, SPLIT, true, BF, NARROW>(a, phi, J, st);
  return launch_jac_t<C, In, SPLIT, false, BF, NARROW>(a, phi, J, st);
}

// lam[r][s] = sum_d phi[r][dcol0 + d] conj(g[det0_i + d][s]) for the instance i of row r
template <typename T>
__global__ void adjoint_fields_kernel(const T* __restrict__ phi, int64_t nn, int64_t ld, int64_t dcol0,
                                      const T* __restrict__ g, int64_t ns, const int64_t* __restrict__ row0,
                                      const int64_t* __restrict__ det0, int64_t ninst, T* __restrict__ lam) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nn * ns;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = t / ns, s = t - r * ns;
    int64_t lo = 0, hi = ninst - 1;  // instance of row r: row0[i] <= r < row0[i + 1]
    while (lo < hi) {
      const int64_t mid = (lo + hi + 1) >> 1;
      if (row0[mid] <= r) lo = mid; else hi = mid - 1;
    }
    const int64_t d0 = det0[lo], nd = det0[lo + 1] - d0;
    T acc = s_zero(T());
    for (int64_t d = 0; d < nd; ++d) {
      T gv = g[(d0 + d) * ns + s];
      if constexpr (Scalar<T>::is_complex) gv.y = -gv.y;
      acc = s_fma(phi[r * ld + dcol0 + d], gv, acc);
    }
    lam[r * ns + s] = acc;
  }
}

}  // namespace rb

using namespace rb;

extern "C" {

int rb_adjoint_fields(const void* phi, int64_t nn, int64_t ld, int64_t dcol0, const void* g, int64_t ns,
                      const int64_t* row0, const int64_t* det0, int64_t ninst, int32_t kind, void* lam,
                      void* stream) {
  if (!phi || !g || !row0 || !det0 || !lam || nn < 0 || ns < 0 || ninst < 1 || dcol0 < 0 || dcol0 > ld)
    return fail(RB_EARG, "rb_adjoint_fields: bad arguments");
  if (nn * ns == 0) return RB_OK;
  const unsigned grid = (unsigned)std::min<int64_t>(ceil_div(nn * ns, 256), 148 * 32);
  cudaStream_t st = as_stream(stream);
  if (kind == RB_F64)
    adjoint_fields_kernel<double><<<grid, 256, 0, st>>>((const double*)phi, nn, ld, dcol0, (const double*)g, ns, row0,
                                                        det0, ninst, (double*)lam);
  else if (kind == RB_C128)
    adjoint_fields_kernel<cdouble><<<grid, 256, 0, st>>>((const cdouble*)phi, nn, ld, dcol0, (const cdouble*)g, ns,
                                                         row0, det0, ninst, (cdouble*)lam);
  else
    return fail(RB_EARG, "rb_adjoint_fields: kind must be RB_F64 or RB_C128");
  RB_LAUNCH_CHECK();
  return RB_OK;
}


int rb_jac_range(const rb_mesh* mesh, int32_t what, const void* phi, int32_t phi_kind, int64_t ld,
                 const int32_t* cols, int32_t nc, int32_t det0, int32_t ndet, const int32_t* pair_src,
                 const int32_t* pair_det, int64_t nsd, void* J, int64_t ldj, int32_t out_kind, int32_t rmax,
                 int32_t emax, const double* evol, const double* ddd, int64_t node0, int64_t count,
                 void* stream) {
  if (!mesh || !phi || !cols || !pair_src || !pair_det || !J || !evol) return fail(RB_EARG, "rb_jac: null argument");
  if (what == JAC_D && !ddd) return fail(RB_EARG, "rb_jac: RB_JAC_D needs deldotdel");
  if (what < JAC_MUA_REF || what > JAC_D) return fail(RB_EARG, "rb_jac: bad quantity");
  if (node0 < 0 || count < 0 || node0 + count > mesh->nn) return fail(RB_EARG, "rb_jac: node range outside the mesh");
  if (nc < 1 || ndet < 1 || det0 < 0 || det0 + ndet > nc || ldj < count)
    return fail(RB_EARG, "rb_jac: bad column map");
  if (rmax < 1 || rmax > 64 || emax < 1 || emax > 256) return fail(RB_ESIZE, "rb_jac: rmax/emax out of range");
  if (nsd == 0 || count == 0) return RB_OK;
  JacArgs a{mesh->indptr, mesh->indices, mesh->node_eptr, mesh->node_elist, mesh->elem, evol, ddd, node0 + count,
            cols, nc, det0, ndet, pair_src, pair_det, nsd, ld, ldj, rmax, emax, what, 0, node0};
  // the blocked path needs the full detector-major grid of sources x detectors
  // with both counts multiple of 4; the caller flags it through nsd < 0
  if (nsd < 0) {
    a.nsd = -nsd;
    if (a.nsd != (int64_t)det0 * ndet || det0 % 4 || ndet % 4)
      return fail(RB_EARG, "rb_jac: grid pair layout needs nsd = nsrc * ndet with both multiples of 4");
    a.grid = 1;
  }
  cudaStream_t st = as_stream(stream);
  const bool cin = (phi_kind == RB_C128 || phi_kind == RB_C64);
  if (out_kind == RB_JAC_SPLIT_F32_ACC64) {  // FP32 rows of products formed in FP64
    if (!cin) return fail(RB_EARG, "rb_jac: split output needs complex phi");
    return phi_kind == RB_C64 ? launch_jac<cdouble, cfloat, true, false, true>(a, phi, J, st)
                              : launch_jac<cdouble, cdouble, true, false, true>(a, phi, J, st);
  }
  if (out_kind == RB_JAC_F32_ACC64) {
    if (cin) return fail(RB_EARG, "rb_jac: RB_JAC_F32_ACC64 needs real phi (complex: RB_JAC_SPLIT_F32_ACC64)");
    return phi_kind == RB_F32 ? launch_jac<double, float, false, false, true>(a, phi, J, st)
                              : launch_jac<double, double, false, false, true>(a, phi, J, st);
  }
  if (out_kind == RB_JAC_SPLIT_BF16) {
    if (!cin) return fail(RB_EARG, "rb_jac: split output needs complex phi");
    return phi_kind == RB_C64 ? launch_jac<cfloat, cfloat, true, true>(a, phi, J, st)
                              : launch_jac<cfloat, cdouble, true, true>(a, phi, J, st);
  }
  if (out_kind == RB_JAC_BF16) {
    if (cin) return fail(RB_EARG, "rb_jac: BF16 rows need real phi (complex phi: RB_JAC_SPLIT_BF16)");
    return phi_kind == RB_F32 ? launch_jac<float, float, false, true>(a, phi, J, st)
                              : launch_jac<float, double, false, true>(a, phi, J, st);
  }
  if (out_kind == RB_JAC_SPLIT_F32 || out_kind == RB_JAC_SPLIT_F64) {
    if (!cin) return fail(RB_EARG, "rb_jac: split output needs complex phi");
    if (out_kind == RB_JAC_SPLIT_F32)
      return phi_kind == RB_C64 ? launch_jac<cfloat, cfloat, true>(a, phi, J, st)
                                : launch_jac<cfloat, cdouble, true>(a, phi, J, st);
    return phi_kind == RB_C64 ? launch_jac<cdouble, cfloat, true>(a, phi, J, st)
                              : launch_jac<cdouble, cdouble, true>(a, phi, J, st);
  }
  const bool cout = (out_kind == RB_C128 || out_kind == RB_C64);
  if (cin != cout) return fail(RB_EARG, "rb_jac: complex phi needs a complex output kind and vice versa");
  switch (out_kind * 4 + phi_kind) {
    case RB_F32 * 4 + RB_F32: return launch_jac<float, float>(a, phi, J, st);
    case RB_F32 * 4 + RB_F64: return launch_jac<float, double>(a, phi, J, st);
    case RB_F64 * 4 + RB_F32: return launch_jac<double, float>(a, phi, J, st);
    case RB_F64 * 4 + RB_F64: return launch_jac<double, double>(a, phi, J, st);
    case RB_C64 * 4 + RB_C64: return launch_jac<cfloat, cfloat>(a, phi, J, st);
    case RB_C64 * 4 + RB_C128: return launch_jac<cfloat, cdouble>(a, phi, J, st);
    case RB_C128 * 4 + RB_C64: return launch_jac<cdouble, cfloat>(a, phi, J, st);
    case RB_C128 * 4 + RB_C128: return launch_jac<cdouble, cdouble>(a, phi, J, st);
    default: return fail(RB_EARG, "rb_jac: bad kinds");
  }
}

int rb_jac(const rb_mesh* mesh, int32_t what, const void* phi, int32_t phi_kind, int64_t ld,
           const int32_t* cols, int32_t nc, int32_t det0, int32_t ndet, const int32_t* pair_src,
           const int32_t* pair_det, int64_t nsd, void* J, int64_t ldj, int32_t out_kind, int32_t rmax,
           int32_t emax, const double* evol, const double* ddd, void* stream) {
  if (!mesh) return fail(RB_EARG, "rb_jac: null argument");
  return rb_jac_range(mesh, what, phi, phi_kind, ld, cols, nc, det0, ndet, pair_src, pair_det, nsd, J, ldj,
                      out_kind, rmax, emax, evol, ddd, 0, mesh->nn, stream);
}

int rb_jac_tensor_cores(int32_t on) {
  g_jac_tc_on = on != 0;
  return RB_OK;
}

int rb_jac_status(void* stream) {
  cudaStream_t st = as_stream(stream);
  RB_CUDA_TRY(cudaStreamSynchronize(st));
  int h = 0;
  RB_CUDA_TRY(cudaMemcpyFromSymbol(&h, g_jac_tc_err, sizeof(int)));
  if (h) {
    const int zero = 0;
    RB_CUDA_TRY(cudaMemcpyToSymbol(g_jac_tc_err, &zero, sizeof(int)));
    return fail(RB_ECUDA, "rb_jac: a tensor-core wait gave up (code %d); the rows are not valid", h);
  }
  return RB_OK;
}

int rb_jac_elem(const rb_mesh* mesh, const double* evol, const void* phi, int32_t phi_kind, int64_t ld,
                const int32_t* src_col, const int32_t* det_col, int64_t nsd, void* je, void* stream) {
  if (!mesh || !evol || !phi || !src_col || !det_col || !je) return fail(RB_EARG, "rb_jac_elem: null argument");
  if (nsd == 0 || mesh->ne == 0) return RB_OK;
  const unsigned g = (unsigned)std::min<int64_t>(ceil_div(nsd * mesh->ne, 256), 148 * 32);
  cudaStream_t st = as_stream(stream);
  if (phi_kind == RB_F64)
    jac_elem_kernel<double><<<g, 256, 0, st>>>(evol, mesh->elem, mesh->ne, (const double*)phi, ld, src_col,
                                               det_col, nsd, (double*)je);
  else if (phi_kind == RB_C128)
    jac_elem_kernel<cdouble><<<g, 256, 0, st>>>(evol, mesh->elem, mesh->ne, (const cdouble*)phi, ld,
                                                src_col, det_col, nsd, (cdouble*)je);
  else
    return fail(RB_EARG, "rb_jac_elem: phi kind must be RB_F64 or RB_C128");
  RB_LAUNCH_CHECK();
  return RB_OK;
}

}  // extern "C"
