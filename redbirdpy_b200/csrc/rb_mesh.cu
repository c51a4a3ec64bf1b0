// Mesh-side kernels: scans, node->cell incidence, the CSR sparsity pattern,
// element gradients (deldotdel), point location, point-optode RHS and the
// detector readout.
#include <algorithm>

#include "rb_common.cuh"

namespace rb {

std::string& last_error() {
  static thread_local std::string msg;
  return msg;
}

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  last_error() = buf;
  return code;
}

// ------------------------------------------------------------------- scan
// Three-phase exclusive scan of int32 counts: per-block scan of kScanItems
// items, recursive scan of the block totals, then a uniform add.
constexpr int kScanThreads = 512;
constexpr int kScanPer = 8;
constexpr int kScanItems = kScanThreads * kScanPer;

__global__ void scan_block_kernel(const int32_t* __restrict__ in, int32_t* __restrict__ out,
                                  int64_t n, int32_t* __restrict__ block_tot) {
  __shared__ int32_t warp_tot[kScanThreads / kWarp];
  const int64_t base = (int64_t)blockIdx.x * kScanItems + (int64_t)threadIdx.x * kScanPer;
  int32_t v[kScanPer];
  int32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    v[k] = (base + k < n) ? in[base + k] : 0;
    s += v[k];
  }
  // inclusive warp scan of per-thread sums
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int32_t inc = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int32_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) warp_tot[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    int32_t w = (lane < kScanThreads / kWarp) ? warp_tot[lane] : 0;
    int32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int32_t t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    if (lane < kScanThreads / kWarp) warp_tot[lane] = wi - w;  // exclusive
    if (lane == kScanThreads / kWarp - 1) block_tot[blockIdx.x] = wi;
  }
  __syncthreads();
  int32_t run = warp_tot[wid] + inc - s;
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
}

__global__ void scan_add_kernel(int32_t* __restrict__ out, int64_t n,
                                const int32_t* __restrict__ block_off) {
  const int64_t i = (int64_t)blockIdx.x * kScanItems + threadIdx.x;
  const int32_t add = block_off[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    int64_t j = i + (int64_t)k * kScanThreads;
    if (j < n) out[j] += add;
  }
}

size_t scan_work_bytes(int64_t n) {
  size_t total = 0;
  int64_t m = n;
  while (true) {
    int64_t nb = ceil_div(m, kScanItems);
    total += (size_t)(nb + 1) * 2 * sizeof(int32_t);
    if (nb <= 1) break;
    m = nb;
  }
  return total + 256;
}

// out[0..n]: out[i] = sum(in[0..i)), out[n] = total
int scan_exclusive(const int32_t* in, int32_t* out, int64_t n, void* work, size_t work_bytes,
                   cudaStream_t st) {
  if (work_bytes < scan_work_bytes(n)) return fail(RB_EARG, "scan workspace too small");
  int64_t nb = ceil_div(n, kScanItems);
  if (nb == 0) {
    RB_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(int32_t), st));
    return RB_OK;
  }
  int32_t* tot = reinterpret_cast<int32_t*>(work);
  int32_t* off = tot + nb + 1;
  scan_block_kernel<<<(unsigned)nb, kScanThreads, 0, st>>>(in, out, n, tot);
  RB_LAUNCH_CHECK();
  if (nb > 1) {
    RB_TRY(scan_exclusive(tot, off, nb, off + nb + 1,
                          work_bytes - (size_t)(2 * (nb + 1)) * sizeof(int32_t), st));
    scan_add_kernel<<<(unsigned)nb, kScanThreads, 0, st>>>(out, n, off);
    RB_LAUNCH_CHECK();
    // total = off[nb]
    RB_CUDA_TRY(cudaMemcpyAsync(out + n, off + nb, sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
  } else {
    RB_CUDA_TRY(cudaMemcpyAsync(out + n, tot, sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
  }
  return RB_OK;
}

// -------------------------------------------------------------- incidence
__global__ void inc_count_kernel(const int32_t* __restrict__ cells, int64_t total,
                                 int32_t* __restrict__ cnt) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&cnt[cells[t]], 1);
}

__global__ void inc_scatter_kernel(const int32_t* __restrict__ cells, int32_t nv, int64_t total,
                                   const int32_t* __restrict__ ptr, int32_t* __restrict__ fill,
                                   int32_t* __restrict__ tmp) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int32_t nd = cells[t];
    int32_t pos = atomicAdd(&fill[nd], 1);
    tmp[ptr[nd] + pos] = (int32_t)(t / nv);
  }
}

// warp per node: rank-sort the node's (distinct) cell ids from tmp into list
__global__ void inc_sort_kernel(const int32_t* __restrict__ ptr, const int32_t* __restrict__ tmp,
                                int32_t* __restrict__ list, int64_t nn) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t n = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); n < nn; n += warps) {
    const int32_t b = ptr[n], L = ptr[n + 1] - b;
    for (int t = lane; t < L; t += 32) {
      int32_t v = tmp[b + t], r = 0;
      for (int u = 0; u < L; ++u) r += (tmp[b + u] < v);
      list[b + r] = v;
    }
  }
}

// ------------------------------------------------------------ CSR pattern
constexpr int kPatWarps = 8;
constexpr int kPatMaxCand = 1024;  // 4 * (max tets sharing a node)

// Gather the candidate columns of row n (the 4 nodes of every incident tet)
// into smem; returns the count or -1 when the row exceeds the limit.
__device__ __forceinline__ int gather_candidates(const int32_t* __restrict__ elem,
                                                 const int32_t* __restrict__ eptr,
                                                 const int32_t* __restrict__ elist, int64_t n,
                                                 int32_t* cand, int lane) {
  const int32_t b = eptr[n], k = eptr[n + 1] - b;
  if (4 * k > kPatMaxCand) return -1;
  for (int t = lane; t < k; t += 32) {
    int4 e = reinterpret_cast<const int4*>(elem)[elist[b + t]];
    cand[4 * t + 0] = e.x;
    cand[4 * t + 1] = e.y;
    cand[4 * t + 2] = e.z;
    cand[4 * t + 3] = e.w;
  }
  __syncwarp();
  return 4 * k;
}

__global__ void pattern_count_kernel(const int32_t* __restrict__ elem, int64_t nn,
                                     const int32_t* __restrict__ eptr,
                                     const int32_t* __restrict__ elist, int32_t* __restrict__ cnt,
                                     int32_t* __restrict__ err) {
  __shared__ int32_t sc[kPatWarps][kPatMaxCand];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t warps = (int64_t)gridDim.x * kPatWarps;
  for (int64_t n = blockIdx.x * (int64_t)kPatWarps + w; n < nn; n += warps) {
    int m = gather_candidates(elem, eptr, elist, n, sc[w], lane);
    if (m < 0) {
      if (lane == 0) atomicExch(err, 1);
      if (lane == 0) cnt[n] = 0;
      continue;
    }
    int c = 0;
    for (int t = lane; t < m; t += 32) {
      int32_t v = sc[w][t];
      bool first = true;
      for (int u = 0; u < t; ++u)
        if (sc[w][u] == v) { first = false; break; }
      c += first;
    }
    c = warp_sum_i(c);
    if (lane == 0) cnt[n] = c;
    __syncwarp();
  }
}

__global__ void pattern_fill_kernel(const int32_t* __restrict__ elem, int64_t nn,
                                    const int32_t* __restrict__ eptr,
                                    const int32_t* __restrict__ elist,
                                    const int32_t* __restrict__ indptr,
                                    int32_t* __restrict__ indices) {
  __shared__ int32_t sc[kPatWarps][kPatMaxCand];
  __shared__ int8_t sf[kPatWarps][kPatMaxCand];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t warps = (int64_t)gridDim.x * kPatWarps;
  for (int64_t n = blockIdx.x * (int64_t)kPatWarps + w; n < nn; n += warps) {
    int m = gather_candidates(elem, eptr, elist, n, sc[w], lane);
    if (m < 0) continue;
    // first-occurrence flags: each distinct column is represented once
    for (int t = lane; t < m; t += 32) {
      int32_t v = sc[w][t];
      int8_t first = 1;
      for (int u = 0; u < t; ++u)
        if (sc[w][u] == v) { first = 0; break; }
      sf[w][t] = first;
    }
    __syncwarp();
    // rank of each distinct column among the distinct columns of the row
    const int32_t base = indptr[n];
    for (int t = lane; t < m; t += 32) {
      if (!sf[w][t]) continue;
      const int32_t v = sc[w][t];
      int r = 0;
      for (int u = 0; u < m; ++u) r += (sf[w][u] && sc[w][u] < v);
      indices[base + r] = v;
    }
    __syncwarp();
  }
}

// --------------------------------------------------------------- gradients
// cofactor vectors c_j = 6V * grad(lambda_j) and the signed 6V of a tet
__device__ __forceinline__ void tet_cofactors(const double* __restrict__ node, int4 e, double c[4][3],
                                              double& det6) {
  const double* p0 = node + 3 * (int64_t)e.x;
  const double* p1 = node + 3 * (int64_t)e.y;
  const double* p2 = node + 3 * (int64_t)e.z;
  const double* p3 = node + 3 * (int64_t)e.w;
  double a[3], b[3], d[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    a[k] = p1[k] - p0[k];
    b[k] = p2[k] - p0[k];
    d[k] = p3[k] - p0[k];
  }
  // c1 = b x d, c2 = d x a, c3 = a x b, c0 = -(c1+c2+c3)
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

__global__ void deldotdel_kernel(const double* __restrict__ node, const int32_t* __restrict__ elem,
                                 int64_t ne, double* __restrict__ ddd, double* __restrict__ evol) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne;
       e += (int64_t)gridDim.x * blockDim.x) {
    int4 en = reinterpret_cast<const int4*>(elem)[e];
    double c[4][3], det6;
    tet_cofactors(node, en, c, det6);
    const double s = 1.0 / (6.0 * fabs(det6));  // 1/(36 V)
    if (evol) evol[e] = fabs(det6) * (1.0 / 6.0);
    int k = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = i; j < 4; ++j)
        ddd[e * 10 + (k++)] = (c[i][0] * c[j][0] + c[i][1] * c[j][1] + c[i][2] * c[j][2]) * s;
  }
}

// --------------------------------------------------------- point location
constexpr double kBaryTol = 1e-9;

__device__ __forceinline__ double det3(const double* a, const double* b, const double* c) {
  return a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) +
         a[2] * (b[0] * c[1] - b[1] * c[0]);
}

__device__ __forceinline__ void tet_bary(const double* __restrict__ node, int4 e, const double* p,
                                         double lam[4]) {
  const double* x0 = node + 3 * (int64_t)e.x;
  const double* x1 = node + 3 * (int64_t)e.y;
  const double* x2 = node + 3 * (int64_t)e.z;
  const double* x3 = node + 3 * (int64_t)e.w;
  double a[3], b[3], c[3], q[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    a[k] = x1[k] - x0[k];
    b[k] = x2[k] - x0[k];
    c[k] = x3[k] - x0[k];
    q[k] = p[k] - x0[k];
  }
  const double v = det3(a, b, c);
  lam[1] = det3(q, b, c) / v;
  lam[2] = det3(a, q, c) / v;
  lam[3] = det3(a, b, q) / v;
  lam[0] = 1.0 - lam[1] - lam[2] - lam[3];
}

__global__ void tsearch_kernel(const double* __restrict__ node, const int32_t* __restrict__ elem,
                               int64_t ne, const double* __restrict__ pts, int64_t npts,
                               int32_t* __restrict__ best) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne;
       e += (int64_t)gridDim.x * blockDim.x) {
    int4 en = reinterpret_cast<const int4*>(elem)[e];
    double lo[3], hi[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      double x0 = node[3 * (int64_t)en.x + k], x1 = node[3 * (int64_t)en.y + k];
      double x2 = node[3 * (int64_t)en.z + k], x3 = node[3 * (int64_t)en.w + k];
      lo[k] = fmin(fmin(x0, x1), fmin(x2, x3)) - 1e-9;
      hi[k] = fmax(fmax(x0, x1), fmax(x2, x3)) + 1e-9;
    }
    for (int64_t k = 0; k < npts; ++k) {
      const double* p = pts + 3 * k;
      if (p[0] < lo[0] || p[0] > hi[0] || p[1] < lo[1] || p[1] > hi[1] || p[2] < lo[2] ||
          p[2] > hi[2])
        continue;
      double lam[4];
      tet_bary(node, en, p, lam);
      if (lam[0] >= -kBaryTol && lam[1] >= -kBaryTol && lam[2] >= -kBaryTol && lam[3] >= -kBaryTol)
        atomicMin(&best[k], (int32_t)e);
    }
  }
}

__global__ void tsearch_bary_kernel(const double* __restrict__ node, const int32_t* __restrict__ elem,
                                    const double* __restrict__ pts, int64_t npts,
                                    int32_t* __restrict__ loc, double* __restrict__ bary) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= npts) return;
  int32_t e = loc[k];
  if (e == 0x7fffffff) {
    loc[k] = -1;
    for (int m = 0; m < 4; ++m) bary[4 * k + m] = __longlong_as_double(0x7ff8000000000000ull);
    return;
  }
  double lam[4];
  tet_bary(node, reinterpret_cast<const int4*>(elem)[e], pts + 3 * k, lam);
  for (int m = 0; m < 4; ++m) bary[4 * k + m] = lam[m];
}

__global__ void point_rhs_kernel(const int32_t* __restrict__ elem, const int32_t* __restrict__ loc,
                                 const double* __restrict__ bary, int64_t npts, int64_t ld,
                                 int64_t col0, double* __restrict__ B) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= npts || loc[k] < 0) return;
  int4 e = reinterpret_cast<const int4*>(elem)[loc[k]];
  const int32_t nd[4] = {e.x, e.y, e.z, e.w};
  // nodes of a tet are distinct: plain stores, no accumulation needed
  for (int m = 0; m < 4; ++m) B[(int64_t)nd[m] * ld + col0 + k] = bary[4 * k + m];
}

template <typename T>
__global__ void getdet_kernel(const int32_t* __restrict__ elem, const int32_t* __restrict__ loc,
                              const double* __restrict__ bary, int64_t ndet,
                              const T* __restrict__ phi, int64_t ld, int64_t nsrc,
                              T* __restrict__ det) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= ndet * nsrc) return;
  int64_t d = t / nsrc, s = t % nsrc;
  T acc = s_zero(T());
  if (loc[d] >= 0) {
    int4 e = reinterpret_cast<const int4*>(elem)[loc[d]];
    const int32_t nd[4] = {e.x, e.y, e.z, e.w};
    for (int m = 0; m < 4; ++m) {
      T w = s_zero(T());
      if constexpr (Scalar<T>::is_complex) w.x = bary[4 * d + m];
      else w = bary[4 * d + m];
      acc = s_fma(w, phi[(int64_t)nd[m] * ld + s], acc);
    }
  }
  det[t] = acc;
}

__global__ void fill_i32_kernel(int32_t* __restrict__ p, int64_t n, int32_t v) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

}  // namespace rb

using namespace rb;

extern "C" {

const char* rb_last_error(void) { return rb::last_error().c_str(); }
int rb_version(void) { return 1; }

size_t rb_incidence_work_bytes(int64_t ncell, int32_t nv, int64_t nn) {
  return (size_t)nn * 4 + (size_t)ncell * nv * 4 + scan_work_bytes(nn) + 512;
}

int rb_incidence(const int32_t* cells, int32_t nv, int64_t ncell, int64_t nn, int32_t* ptr,
                 int32_t* list, void* work, size_t work_bytes, void* stream) {
  if (!cells || !ptr || !list || nv < 1 || ncell < 0 || nn < 1)
    return fail(RB_EARG, "rb_incidence: bad arguments");
  if (ncell * nv >= (int64_t)0x7fffffff) return fail(RB_ESIZE, "rb_incidence: too many cells");
  if (work_bytes < rb_incidence_work_bytes(ncell, nv, nn))
    return fail(RB_EARG, "rb_incidence: workspace too small");
  cudaStream_t st = as_stream(stream);
  char* w = reinterpret_cast<char*>(work);
  int32_t* cnt = reinterpret_cast<int32_t*>(w);
  w += ((size_t)nn * 4 + 255) / 256 * 256;
  int32_t* tmp = reinterpret_cast<int32_t*>(w);
  w += ((size_t)ncell * nv * 4 + 255) / 256 * 256;
  size_t scan_bytes = work_bytes - (size_t)(w - reinterpret_cast<char*>(work));
  const int64_t total = ncell * nv;
  RB_CUDA_TRY(cudaMemsetAsync(cnt, 0, nn * 4, st));
  unsigned g = (unsigned)std::min<int64_t>(ceil_div(std::max<int64_t>(total, 1), 256), 148 * 32);
  inc_count_kernel<<<g, 256, 0, st>>>(cells, total, cnt);
  RB_LAUNCH_CHECK();
  RB_TRY(scan_exclusive(cnt, ptr, nn, w, scan_bytes, st));
  RB_CUDA_TRY(cudaMemsetAsync(cnt, 0, nn * 4, st));
  inc_scatter_kernel<<<g, 256, 0, st>>>(cells, nv, total, ptr, cnt, tmp);
  RB_LAUNCH_CHECK();
  unsigned gs = (unsigned)std::min<int64_t>(ceil_div(nn, 8), 148 * 64);
  inc_sort_kernel<<<gs, 256, 0, st>>>(ptr, tmp, list, nn);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

size_t rb_csr_pattern_work_bytes(int64_t nn) { return (size_t)nn * 4 + 256 + 16 + scan_work_bytes(nn); }

int rb_csr_pattern_count(const int32_t* elem, int64_t nn, const int32_t* eptr, const int32_t* elist,
                         int32_t* indptr, void* work, size_t work_bytes, void* stream) {
  if (!elem || !eptr || !elist || !indptr || nn < 1) return fail(RB_EARG, "rb_csr_pattern_count: bad arguments");
  if (work_bytes < rb_csr_pattern_work_bytes(nn)) return fail(RB_EARG, "rb_csr_pattern_count: workspace too small");
  cudaStream_t st = as_stream(stream);
  char* w = reinterpret_cast<char*>(work);
  int32_t* cnt = reinterpret_cast<int32_t*>(w);
  w += ((size_t)nn * 4 + 255) / 256 * 256;
  int32_t* err = reinterpret_cast<int32_t*>(w);
  w += 16;
  RB_CUDA_TRY(cudaMemsetAsync(err, 0, 4, st));
  unsigned g = (unsigned)std::min<int64_t>(ceil_div(nn, kPatWarps), 148 * 16);
  pattern_count_kernel<<<g, kPatWarps * 32, 0, st>>>(elem, nn, eptr, elist, cnt, err);
  RB_LAUNCH_CHECK();
  RB_TRY(scan_exclusive(cnt, indptr, nn, w, work_bytes - (size_t)(w - reinterpret_cast<char*>(work)), st));
  int32_t herr = 0;
  RB_CUDA_TRY(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, st));
  RB_CUDA_TRY(cudaStreamSynchronize(st));
  if (herr) return fail(RB_ESIZE, "rb_csr_pattern_count: a node belongs to more than %d tets", kPatMaxCand / 4);
  return RB_OK;
}

int rb_csr_pattern_fill(const int32_t* elem, int64_t nn, const int32_t* eptr, const int32_t* elist,
                        const int32_t* indptr, int32_t* indices, void* stream) {
  if (!elem || !eptr || !elist || !indptr || !indices) return fail(RB_EARG, "rb_csr_pattern_fill: bad arguments");
  cudaStream_t st = as_stream(stream);
  unsigned g = (unsigned)std::min<int64_t>(ceil_div(nn, kPatWarps), 148 * 16);
  pattern_fill_kernel<<<g, kPatWarps * 32, 0, st>>>(elem, nn, eptr, elist, indptr, indices);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

int rb_deldotdel(const double* node, const int32_t* elem, int64_t ne, double* ddd, double* evol, void* stream) {
  if (!node || !elem || !ddd || ne < 0) return fail(RB_EARG, "rb_deldotdel: bad arguments");
  if (ne == 0) return RB_OK;
  unsigned g = (unsigned)std::min<int64_t>(ceil_div(ne, 256), 148 * 32);
  deldotdel_kernel<<<g, 256, 0, as_stream(stream)>>>(node, elem, ne, ddd, evol);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

int rb_tsearch(const double* node, const int32_t* elem, int64_t ne, const double* pts, int64_t npts,
               int32_t* loc, double* bary, void* stream) {
  if (!node || !elem || !pts || !loc || !bary || ne < 1 || npts < 0)
    return fail(RB_EARG, "rb_tsearch: bad arguments");
  if (npts == 0) return RB_OK;
  cudaStream_t st = as_stream(stream);
  fill_i32_kernel<<<(unsigned)ceil_div(npts, 256), 256, 0, st>>>(loc, npts, 0x7fffffff);
  RB_LAUNCH_CHECK();
  unsigned g = (unsigned)std::min<int64_t>(ceil_div(ne, 256), 148 * 32);
  tsearch_kernel<<<g, 256, 0, st>>>(node, elem, ne, pts, npts, loc);
  RB_LAUNCH_CHECK();
  tsearch_bary_kernel<<<(unsigned)ceil_div(npts, 128), 128, 0, st>>>(node, elem, pts, npts, loc, bary);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

int rb_point_rhs(const int32_t* elem, const int32_t* loc, const double* bary, int64_t npts,
                 int64_t nn, int64_t ld, int64_t col0, double* B, void* stream) {
  if (!elem || !loc || !bary || !B || npts < 0 || nn < 1 || col0 < 0 || col0 + npts > ld)
    return fail(RB_EARG, "rb_point_rhs: bad arguments");
  if (npts == 0) return RB_OK;
  point_rhs_kernel<<<(unsigned)ceil_div(npts, 128), 128, 0, as_stream(stream)>>>(elem, loc, bary, npts,
                                                                                 ld, col0, B);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

int rb_femgetdet(const int32_t* elem, const int32_t* loc_det, const double* bary_det, int64_t ndet,
                 const void* phi, int64_t ld, int64_t nsrc, int32_t kind, void* detval, void* stream) {
  if (!elem || !loc_det || !bary_det || !phi || !detval || ndet < 0 || nsrc < 0 || nsrc > ld)
    return fail(RB_EARG, "rb_femgetdet: bad arguments");
  if (ndet * nsrc == 0) return RB_OK;
  unsigned g = (unsigned)ceil_div(ndet * nsrc, 256);
  cudaStream_t st = as_stream(stream);
  if (kind == RB_F64)
    getdet_kernel<double><<<g, 256, 0, st>>>(elem, loc_det, bary_det, ndet, (const double*)phi, ld,
                                             nsrc, (double*)detval);
  else if (kind == RB_C128)
    getdet_kernel<cdouble><<<g, 256, 0, st>>>(elem, loc_det, bary_det, ndet, (const cdouble*)phi, ld,
                                              nsrc, (cdouble*)detval);
  else
    return fail(RB_EARG, "rb_femgetdet: kind must be RB_F64 or RB_C128");
  RB_LAUNCH_CHECK();
  return RB_OK;
}

}  // extern "C"
