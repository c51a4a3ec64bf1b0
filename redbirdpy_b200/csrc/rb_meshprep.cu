// Mesh preparation on the device (meshprep, redbirdpy/utility.py:101-246,
// with the reference's own fallbacks for a missing iso2mesh):
//   rb_reorient     swap nodes 0 and 1 of every tet of negative signed volume
//                   (_meshreorient_fallback, utility.py:1047-1063) and write
//                   |V| (_elemvolume_fallback, utility.py:1090-1109);
//   rb_volface      boundary triangles: the 4 faces of every tet (node orders
//                   (0,2,1), (0,1,3), (0,3,2), (1,2,3)), keyed by their sorted
//                   node triple, sorted (radix sort), the keys that occur once
//                   kept with the owning tet's orientation, in key order --
//                   np.unique's order in _volface_fallback (utility.py:1066-1087);
//   rb_face_area    triangle areas (_elemvolume_fallback);
//   rb_nodevolume   a quarter of the incident tets' volumes per node, summed
//                   in ascending tet order (np.bincount's order, utility.py:1005-1017).
// The arithmetic is written without fused multiply-adds, in numpy's order of
// operations, so that volumes and areas carry the same bits as the host's.
#include <algorithm>

#include <cub/cub.cuh>

#include "rb_common.cuh"

namespace rb {

// (b - a) x (c - a) . (d - a), as numpy's cross then a left-to-right sum
__device__ __forceinline__ double signed6(const double* __restrict__ node, int32_t a, int32_t b, int32_t c,
                                          int32_t d) {
  const double* p0 = node + 3 * (int64_t)a;
  const double* p1 = node + 3 * (int64_t)b;
  const double* p2 = node + 3 * (int64_t)c;
  const double* p3 = node + 3 * (int64_t)d;
  const double u0 = __dsub_rn(p1[0], p0[0]), u1 = __dsub_rn(p1[1], p0[1]), u2 = __dsub_rn(p1[2], p0[2]);
  const double v0 = __dsub_rn(p2[0], p0[0]), v1 = __dsub_rn(p2[1], p0[1]), v2 = __dsub_rn(p2[2], p0[2]);
  const double w0 = __dsub_rn(p3[0], p0[0]), w1 = __dsub_rn(p3[1], p0[1]), w2 = __dsub_rn(p3[2], p0[2]);
  const double c0 = __dsub_rn(__dmul_rn(u1, v2), __dmul_rn(u2, v1));
  const double c1 = __dsub_rn(__dmul_rn(u2, v0), __dmul_rn(u0, v2));
  const double c2 = __dsub_rn(__dmul_rn(u0, v1), __dmul_rn(u1, v0));
  return __dadd_rn(__dadd_rn(__dmul_rn(c0, w0), __dmul_rn(c1, w1)), __dmul_rn(c2, w2));
}

__global__ void reorient_kernel(const double* __restrict__ node, int32_t* __restrict__ elem, int64_t ne,
                                double* __restrict__ evol, int32_t* __restrict__ flipped) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne; e += (int64_t)gridDim.x * blockDim.x) {
    int4 t = reinterpret_cast<int4*>(elem)[e];
    if (signed6(node, t.x, t.y, t.z, t.w) < 0.0) {
      const int32_t s = t.x;
      t.x = t.y;
      t.y = s;
      reinterpret_cast<int4*>(elem)[e] = t;
      if (flipped) atomicAdd(flipped, 1);
    }
    if (evol) evol[e] = __ddiv_rn(fabs(signed6(node, t.x, t.y, t.z, t.w)), 6.0);
  }
}

// the 4 faces of tet e in the reference's order (face f of the stacked
// arrays is tet f % ne, kind f / ne); key = (s0 nn + s1) nn + s2 of the
// sorted triple
__device__ __forceinline__ int3 tet_face(const int32_t* __restrict__ elem, int64_t ne, int64_t f) {
  const int64_t e = f % ne;
  const int kind = (int)(f / ne);
  const int4 t = reinterpret_cast<const int4*>(elem)[e];
  switch (kind) {
    case 0: return make_int3(t.x, t.z, t.y);
    case 1: return make_int3(t.x, t.y, t.w);
    case 2: return make_int3(t.x, t.w, t.z);
    default: return make_int3(t.y, t.z, t.w);
  }
}

__global__ void face_keys_kernel(const int32_t* __restrict__ elem, int64_t ne, int64_t nn, int64_t* __restrict__ key,
                                 int32_t* __restrict__ idx) {
  const int64_t nf = 4 * ne;
  for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < nf; f += (int64_t)gridDim.x * blockDim.x) {
    const int3 v = tet_face(elem, ne, f);
    int64_t a = v.x, b = v.y, c = v.z, s;
    if (a > b) { s = a; a = b; b = s; }
    if (b > c) { s = b; b = c; c = s; }
    if (a > b) { s = a; a = b; b = s; }
    key[f] = (a * nn + b) * nn + c;
    idx[f] = (int32_t)f;
  }
}

// 1 where a sorted key occurs once
__global__ void unique_flag_kernel(const int64_t* __restrict__ key, int64_t n, int32_t* __restrict__ flag) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    flag[i] = (i == 0 || key[i - 1] != key[i]) && (i == n - 1 || key[i + 1] != key[i]);
}

__global__ void face_write_kernel(const int32_t* __restrict__ elem, int64_t ne, const int32_t* __restrict__ idx,
                                  const int32_t* __restrict__ flag, const int32_t* __restrict__ pos, int64_t n,
                                  int32_t* __restrict__ face) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (!flag[i]) continue;
    const int3 v = tet_face(elem, ne, idx[i]);
    const int64_t o = 3 * (int64_t)pos[i];
    face[o] = v.x;
    face[o + 1] = v.y;
    face[o + 2] = v.z;
  }
}

__global__ void face_area_kernel(const double* __restrict__ node, const int32_t* __restrict__ face, int64_t nf,
                                 double* __restrict__ area) {
  for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < nf; f += (int64_t)gridDim.x * blockDim.x) {
    const double* p0 = node + 3 * (int64_t)face[3 * f];
    const double* p1 = node + 3 * (int64_t)face[3 * f + 1];
    const double* p2 = node + 3 * (int64_t)face[3 * f + 2];
    const double u0 = __dsub_rn(p1[0], p0[0]), u1 = __dsub_rn(p1[1], p0[1]), u2 = __dsub_rn(p1[2], p0[2]);
    const double v0 = __dsub_rn(p2[0], p0[0]), v1 = __dsub_rn(p2[1], p0[1]), v2 = __dsub_rn(p2[2], p0[2]);
    const double c0 = __dsub_rn(__dmul_rn(u1, v2), __dmul_rn(u2, v1));
    const double c1 = __dsub_rn(__dmul_rn(u2, v0), __dmul_rn(u0, v2));
    const double c2 = __dsub_rn(__dmul_rn(u0, v1), __dmul_rn(u1, v0));
    const double s = __dadd_rn(__dadd_rn(__dmul_rn(c0, c0), __dmul_rn(c1, c1)), __dmul_rn(c2, c2));
    area[f] = __dmul_rn(0.5, __dsqrt_rn(s));
  }
}

__global__ void nodevolume_kernel(int64_t nn, const int32_t* __restrict__ eptr, const int32_t* __restrict__ elist,
                                  const double* __restrict__ evol, double* __restrict__ nvol) {
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn; n += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int32_t p = eptr[n]; p < eptr[n + 1]; ++p) s = __dadd_rn(s, evol[elist[p]]);
    nvol[n] = __dmul_rn(0.25, s);
  }
}

struct FaceWork {
  int64_t *key, *key2;
  int32_t *idx, *idx2, *flag, *pos;
  void* sort;
  size_t sort_bytes;
  char* scan;
  size_t scan_bytes;
};

static size_t face_carve(char* base, int64_t ne, FaceWork* w) {
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* p = base ? base + off : nullptr;
    off += (bytes + 255) / 256 * 256;
    return p;
  };
  const int64_t n = 4 * ne;
  FaceWork t;
  t.key = (int64_t*)take(8 * n);
  t.key2 = (int64_t*)take(8 * n);
  t.idx = (int32_t*)take(4 * n);
  t.idx2 = (int32_t*)take(4 * n);
  t.flag = (int32_t*)take(4 * (n + 1));
  t.pos = (int32_t*)take(4 * (n + 1));
  t.sort_bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, t.sort_bytes, (const int64_t*)nullptr, (int64_t*)nullptr,
                                  (const int32_t*)nullptr, (int32_t*)nullptr, (int)n);
  t.sort = take(t.sort_bytes);
  t.scan_bytes = scan_work_bytes(n);
  t.scan = take(t.scan_bytes);
  if (w) *w = t;
  return off;
}

}  // namespace rb

using namespace rb;

extern "C" {

int rb_reorient(const double* node, int32_t* elem, int64_t ne, double* evol, int32_t* flipped, void* stream) {
  if (!node || !elem || ne < 0) return fail(RB_EARG, "rb_reorient: bad arguments");
  if (ne == 0) return RB_OK;
  if (reinterpret_cast<uintptr_t>(elem) & 15) return fail(RB_EARG, "rb_reorient: elem must be 16-byte aligned");
  const unsigned g = (unsigned)std::min<int64_t>(ceil_div(ne, 256), 148 * 16);
  reorient_kernel<<<g, 256, 0, as_stream(stream)>>>(node, elem, ne, evol, flipped);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

size_t rb_volface_work_bytes(int64_t ne) {
  if (ne < 1) return 0;
  return face_carve(nullptr, ne, nullptr);
}

int rb_volface(const int32_t* elem, int64_t ne, int64_t nn, int32_t* face, int64_t* nf_out, void* work,
               size_t work_bytes, void* stream) {
  if (!elem || !face || !nf_out || !work || ne < 1 || nn < 1) return fail(RB_EARG, "rb_volface: bad arguments");
  if (nn >= (int64_t(1) << 21)) return fail(RB_ESIZE, "rb_volface: %lld nodes (face keys hold up to 2^21)", (long long)nn);
  if (4 * ne >= (int64_t)0x7fffffff) return fail(RB_ESIZE, "rb_volface: too many tets");
  if (reinterpret_cast<uintptr_t>(elem) & 15) return fail(RB_EARG, "rb_volface: elem must be 16-byte aligned");
  if (work_bytes < rb_volface_work_bytes(ne)) return fail(RB_EARG, "rb_volface: workspace too small");
  cudaStream_t st = as_stream(stream);
  FaceWork w;
  face_carve(reinterpret_cast<char*>(work), ne, &w);
  const int64_t n = 4 * ne;
  const unsigned g = (unsigned)std::min<int64_t>(ceil_div(n, 256), 148 * 32);
  face_keys_kernel<<<g, 256, 0, st>>>(elem, ne, nn, w.key, w.idx);
  RB_LAUNCH_CHECK();
  // stable radix sort: equal keys keep the face order (as np.unique's first index)
  int bits = 1;
  while (bits < 63 && (int64_t(1) << bits) <= nn * nn * nn) ++bits;
  size_t sb = w.sort_bytes;
  RB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(w.sort, sb, w.key, w.key2, w.idx, w.idx2, (int)n, 0, bits, st));
  unique_flag_kernel<<<g, 256, 0, st>>>(w.key2, n, w.flag);
  RB_LAUNCH_CHECK();
  RB_TRY(scan_exclusive(w.flag, w.pos, n, w.scan, w.scan_bytes, st));
  face_write_kernel<<<g, 256, 0, st>>>(elem, ne, w.idx2, w.flag, w.pos, n, face);
  RB_LAUNCH_CHECK();
  int32_t nf = 0;
  RB_CUDA_TRY(cudaMemcpyAsync(&nf, w.pos + n, 4, cudaMemcpyDeviceToHost, st));
  RB_CUDA_TRY(cudaStreamSynchronize(st));
  *nf_out = nf;
  return RB_OK;
}

int rb_face_area(const double* node, const int32_t* face, int64_t nf, double* area, void* stream) {
  if (!node || !face || !area || nf < 0) return fail(RB_EARG, "rb_face_area: bad arguments");
  if (nf == 0) return RB_OK;
  const unsigned g = (unsigned)std::min<int64_t>(ceil_div(nf, 256), 148 * 16);
  face_area_kernel<<<g, 256, 0, as_stream(stream)>>>(node, face, nf, area);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

int rb_nodevolume(int64_t nn, const int32_t* node_eptr, const int32_t* node_elist, const double* evol, double* nvol,
                  void* stream) {
  if (!node_eptr || !node_elist || !evol || !nvol || nn < 1) return fail(RB_EARG, "rb_nodevolume: bad arguments");
  const unsigned g = (unsigned)std::min<int64_t>(ceil_div(nn, 256), 148 * 16);
  nodevolume_kernel<<<g, 256, 0, as_stream(stream)>>>(nn, node_eptr, node_elist, evol, nvol);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

}  // extern "C"
