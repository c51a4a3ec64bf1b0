// FEM matrix assembly (femlhs) into a fixed CSR pattern.
//
// One warp owns one matrix row n.  Its lanes first evaluate, for up to 32
// tets that contain n, the tet's contribution to row n (4 values: the row of
// the local 4x4 stiffness*D + mass*mua (+ i*omega/c*n*mass) block), with the
// P1 gradients recomputed from the node coordinates.  The lanes then switch
// roles and each owns one CSR slot of the row, summing the staged
// contributions whose column matches in ascending tet order, then the Robin
// terms of the row's boundary faces.  No atomics: the result is
// deterministic and written exactly once, FP64 plus an optional FP32 copy,
// together with the reciprocal diagonal used by the Jacobi preconditioner.
#include <algorithm>

#include "rb_common.cuh"

namespace rb {

constexpr int kAsmWarps = 8;

template <bool CPLX> struct AsmVal;
template <> struct AsmVal<false> { typedef double T; typedef float T32; };
template <> struct AsmVal<true> { typedef cdouble T; typedef cfloat T32; };

__device__ __forceinline__ void tet_geometry(const double* __restrict__ node, int4 e, double c[4][3],
                                             double& det6) {
  const double* p0 = node + 3 * (int64_t)e.x;
  const double* p1 = node + 3 * (int64_t)e.y;
  const double* p2 = node + 3 * (int64_t)e.z;
  const double* p3 = node + 3 * (int64_t)e.w;
  double a[3], b[3], d[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double x0 = p0[k];
    a[k] = p1[k] - x0;
    b[k] = p2[k] - x0;
    d[k] = p3[k] - x0;
  }
  c[1][0] = b[1] * d[2] - b[2] * d[1];
  c[1][1] = b[2] * d[0] - b[0] * d[2];
  c[1][2] = b[0] * d[1] - b[1] * d[0];
  c[2][0] = d[1] * a[2] - d[2] * a[1];
  c[2][1] = d[2] * a[0] - d[0] * a[2];
  c[2][2] = d[0] * a[1] - d[1] * a[0];
  c[3][0] = a[1] * b[2] - a[2] * b[1];
  c[3][1] = a[2] * b[0] - a[0] * b[2];
  c[3][2] = a[0] * b[1] - a[1] * b[0];
#pragma unroll
  for (int k = 0; k < 3; ++k) c[0][k] = -(c[1][k] + c[2][k] + c[3][k]);
  det6 = a[0] * c[1][0] + a[1] * c[1][1] + a[2] * c[1][2];
}

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

// Contribution of tet `e` (nodes en) to row `row`: the 4 entries (row, en[j]).
template <bool CPLX, int KIND>
__device__ __forceinline__ void tet_row(const rb_mesh& m, const rb_optics& o, double wc, int64_t e,
                                        int4 en, int64_t row, typename AsmVal<CPLX>::T out[4]) {
  double c[4][3], det6;
  tet_geometry(m.node, en, c, det6);
  const double vol = fabs(det6) * (1.0 / 6.0);
  const double inv36v = 1.0 / (6.0 * fabs(det6));
  const int32_t nd[4] = {en.x, en.y, en.z, en.w};
  int li = 0;
#pragma unroll
  for (int j = 1; j < 4; ++j)
    if (nd[j] == row) li = j;
  double dco, mu[4], msum = 0.0, nr[4], nsum = 0.0;
  const bool nvec = (o.nref != nullptr);
  if (KIND == RB_PROP_NODE) {
    double ds = 0.0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      mu[j] = o.mua[nd[j]];
      msum += mu[j];
      ds += 1.0 / (3.0 * (mu[j] + o.musp[nd[j]]));
      nr[j] = nvec ? o.nref[nd[j]] : o.nref_scalar;
      nsum += nr[j];
    }
    dco = ds * 0.25;
  } else {
    const double ma = o.mua[e];
    dco = 1.0 / (3.0 * (ma + o.musp[e]));
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      mu[j] = ma;
      nr[j] = nvec ? o.nref[e] : o.nref_scalar;
    }
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const double stiff = dco * (c[li][0] * c[j][0] + c[li][1] * c[j][1] + c[li][2] * c[j][2]) * inv36v;
    double mass, imag = 0.0;
    if (KIND == RB_PROP_NODE) {
      // lumped-weight mass of node-based properties: (sum + mu_i + mu_j)/120
      // off the diagonal, (sum + 2 mu_i)/60 on it
      mass = (j == li) ? vol * (msum + 2.0 * mu[li]) * (1.0 / 60.0)
                       : vol * (msum + mu[li] + mu[j]) * (1.0 / 120.0);
      if (CPLX) {
        if (nvec)
          imag = (j == li) ? wc * vol * (nsum + 2.0 * nr[li]) * (1.0 / 60.0)
                           : wc * vol * (nsum + nr[li] + nr[j]) * (1.0 / 120.0);
        else
          imag = wc * o.nref_scalar * ((j == li) ? 0.10 : 0.05) * vol;
      }
    } else {
      mass = ((j == li) ? 0.10 : 0.05) * mu[0] * vol;
      if (CPLX) imag = ((j == li) ? 0.10 : 0.05) * wc * nr[0] * vol;
    }
    put(out[j], stiff + mass, imag);
  }
}

template <bool CPLX, int KIND>
__global__ void __launch_bounds__(kAsmWarps * 32)
femlhs_rows_kernel(rb_mesh m, rb_optics o, double bc, double wc,
                   typename AsmVal<CPLX>::T* __restrict__ val64,
                   typename AsmVal<CPLX>::T32* __restrict__ val32,
                   typename AsmVal<CPLX>::T* __restrict__ dinv64,
                   typename AsmVal<CPLX>::T32* __restrict__ dinv32) {
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
          tet_row<CPLX, KIND>(m, o, wc, e, en, row, v);
          s_nodes[w][lane] = en;
#pragma unroll
          for (int j = 0; j < 4; ++j) s_vals[w][lane][j] = v[j];
        }
        __syncwarp();
        for (int u = 0; u < kc; ++u) {
          const int4 en = s_nodes[w][u];
          const int32_t nd[4] = {en.x, en.y, en.z, en.w};
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            if (nd[j] == col0) acc0 = s_add(acc0, s_vals[w][u][j]);
            if (nd[j] == col1) acc1 = s_add(acc1, s_vals[w][u][j]);
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

template <bool CPLX, int KIND>
int launch_femlhs(const rb_mesh& m, const rb_optics& o, void* v64, void* v32, void* d64, void* d32,
                  cudaStream_t st) {
  typedef typename AsmVal<CPLX>::T T;
  typedef typename AsmVal<CPLX>::T32 T32;
  const double bc = (1.0 - o.reff) / (12.0 * (1.0 + o.reff));
  const double wc = o.omega / kC0;
  unsigned g = (unsigned)std::min<int64_t>(ceil_div(m.nn, kAsmWarps), 148 * 64);
  femlhs_rows_kernel<CPLX, KIND><<<g, kAsmWarps * 32, 0, st>>>(
      m, o, bc, wc, (T*)v64, (T32*)v32, (T*)d64, (T32*)d32);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

}  // namespace rb

using namespace rb;

extern "C" int rb_femlhs(const rb_mesh* mesh, const rb_optics* optics, void* val64, void* val32,
                         void* dinv64, void* dinv32, void* stream) {
  if (!mesh || !optics || !val64) return fail(RB_EARG, "rb_femlhs: mesh, optics and val64 are required");
  const rb_mesh& m = *mesh;
  const rb_optics& o = *optics;
  if (!m.node || !m.elem || !m.indptr || !m.indices || !m.node_eptr || !m.node_elist)
    return fail(RB_EARG, "rb_femlhs: mesh arrays missing");
  if (m.nf > 0 && (!m.face || !m.area || !m.node_fptr || !m.node_flist))
    return fail(RB_EARG, "rb_femlhs: boundary arrays missing");
  if (m.nf == 0 && !m.node_fptr) return fail(RB_EARG, "rb_femlhs: node_fptr required (all zeros when nf == 0)");
  if (!o.mua || !o.musp) return fail(RB_EARG, "rb_femlhs: mua and musp are required");
  if (o.kind != RB_PROP_NODE && o.kind != RB_PROP_ELEM) return fail(RB_EARG, "rb_femlhs: bad property kind");
  if (!(o.omega >= 0.0)) return fail(RB_EARG, "rb_femlhs: omega must be >= 0");
  cudaStream_t st = as_stream(stream);
  const bool cplx = o.omega > 0.0;
  if (cplx)
    return o.kind == RB_PROP_NODE ? launch_femlhs<true, RB_PROP_NODE>(m, o, val64, val32, dinv64, dinv32, st)
                                  : launch_femlhs<true, RB_PROP_ELEM>(m, o, val64, val32, dinv64, dinv32, st);
  return o.kind == RB_PROP_NODE ? launch_femlhs<false, RB_PROP_NODE>(m, o, val64, val32, dinv64, dinv32, st)
                                : launch_femlhs<false, RB_PROP_ELEM>(m, o, val64, val32, dinv64, dinv32, st);
}
