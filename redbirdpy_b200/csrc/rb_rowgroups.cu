// Spatial row groups of the blocked SpMM (rb_spmm_blk.cuh): mesh nodes binned
// into cubes of edge h (about two node spacings, so that a structured grid
// gives 2 x 2 x 2 blocks), each cube's nodes in ascending order cut into
// groups of up to 8 rows, groups in cube order (blocks of 2 x 2 x 2 cubes).  Then, per CSR
// pattern, the union of every group's column lists with a row mask per entry.
// Every step is deterministic: atomics only count or pick scatter slots, and
// each cube's list is re-ranked by node index before it is cut into groups.
#include <algorithm>
#include <cmath>

#include "rb_common.cuh"

namespace rb {

constexpr int kRGRows = 8;

__global__ void rg_bin_kernel(int64_t nn, const double* __restrict__ node, double x0, double y0, double z0, double ih,
                              int32_t nbx, int32_t nby, int32_t nbz, int32_t* __restrict__ key,
                              int32_t* __restrict__ cnt) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x) {
    const double* p = node + 3 * i;
    // NaN coordinates fall into cube 0 (fmax/fmin return the other operand)
    const int bx = (int)fmin(fmax(floor((p[0] - x0) * ih), 0.0), (double)(nbx - 1));
    const int by = (int)fmin(fmax(floor((p[1] - y0) * ih), 0.0), (double)(nby - 1));
    const int bz = (int)fmin(fmax(floor((p[2] - z0) * ih), 0.0), (double)(nbz - 1));
    // cubes numbered in blocks of 2 x 2 x 2 (x fastest inside a block, blocks
    // x fastest): the 8 consecutive groups that the warps of one thread block
    // take together then form a compact 4 x 4 x 4-node block whose column
    // unions overlap in L1 (2% faster SpMM than plain cube order)
    const int sbx = (nbx + 1) >> 1, sby = (nby + 1) >> 1;
    const int32_t b = 8 * ((max(bx, 0) >> 1) + sbx * ((max(by, 0) >> 1) + sby * (max(bz, 0) >> 1))) +
                      (max(bx, 0) & 1) + 2 * (max(by, 0) & 1) + 4 * (max(bz, 0) & 1);
    key[i] = b;
    atomicAdd(cnt + b, 1);
  }
}

// groups per cube: ceil(count / 8)
__global__ void rg_gcount_kernel(int64_t nb, const int32_t* __restrict__ cnt, int32_t* __restrict__ gcnt) {
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < nb; b += (int64_t)gridDim.x * blockDim.x)
    gcnt[b] = (cnt[b] + kRGRows - 1) / kRGRows;
}

__global__ void rg_scatter_kernel(int64_t nn, const int32_t* __restrict__ key, const int32_t* __restrict__ start,
                                  int32_t* __restrict__ fill, int32_t* __restrict__ tmp) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t b = key[i];
    tmp[start[b] + atomicAdd(fill + b, 1)] = (int32_t)i;
  }
}

// one warp per cube: rank its nodes by index, write them into its groups
__global__ void rg_place_kernel(int64_t nb, const int32_t* __restrict__ start, const int32_t* __restrict__ gofs,
                                const int32_t* __restrict__ tmp, int32_t* __restrict__ rows) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t b = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); b < nb; b += warps) {
    const int32_t s = start[b], L = start[b + 1] - s;
    const int64_t g0 = gofs[b];
    for (int t = lane; t < L; t += 32) {
      const int32_t v = tmp[s + t];
      int32_t r = 0;
      for (int u = 0; u < L; ++u) r += (tmp[s + u] < v);
      rows[(g0 + r / kRGRows) * kRGRows + r % kRGRows] = v;
    }
  }
}

// union sizes (count pass) or entries (fill pass) of each group's rows
template <bool FILL>
__global__ void rg_union_kernel(int64_t ng, const int32_t* __restrict__ rows, const int32_t* __restrict__ indptr,
                                const int32_t* __restrict__ indices, int32_t* __restrict__ cnt_or_ptr,
                                int32_t* __restrict__ ucol, uint8_t* __restrict__ umask) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < ng; g += (int64_t)gridDim.x * blockDim.x) {
    int32_t p[kRGRows], e[kRGRows];
#pragma unroll
    for (int r = 0; r < kRGRows; ++r) {
      const int32_t row = rows[g * kRGRows + r];
      p[r] = row >= 0 ? indptr[row] : 0;
      e[r] = row >= 0 ? indptr[row + 1] : 0;
    }
    int32_t c = 0;
    const int32_t out = FILL ? cnt_or_ptr[g] : 0;
    while (true) {
      int32_t m = 0x7fffffff;
#pragma unroll
      for (int r = 0; r < kRGRows; ++r)
        if (p[r] < e[r]) m = min(m, indices[p[r]]);
      if (m == 0x7fffffff) break;
      uint32_t mask = 0;
#pragma unroll
      for (int r = 0; r < kRGRows; ++r)
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

struct RgWork {
  int32_t *key, *cnt, *gcnt, *start, *gofs, *fill, *tmp;
  char* scan;
  size_t scan_bytes;
};

static size_t rg_carve(char* base, int64_t nn, int64_t nb, RgWork* w) {
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* p = base ? base + off : nullptr;
    off += (bytes + 255) / 256 * 256;
    return p;
  };
  RgWork t;
  t.key = (int32_t*)take(4 * nn);
  t.cnt = (int32_t*)take(4 * nb);
  t.gcnt = (int32_t*)take(4 * nb);
  t.start = (int32_t*)take(4 * (nb + 1));
  t.gofs = (int32_t*)take(4 * (nb + 1));
  t.fill = (int32_t*)take(4 * nb);
  t.tmp = (int32_t*)take(4 * nn);
  t.scan_bytes = scan_work_bytes(nb);
  t.scan = take(t.scan_bytes);
  if (w) *w = t;
  return off;
}

}  // namespace rb

using namespace rb;

extern "C" {

size_t rb_rowgroups_work_bytes(int64_t nn, int64_t nbins) {
  if (nn < 1 || nbins < 1) return 0;
  return rg_carve(nullptr, nn, 8 * nbins, nullptr);  // cube slots in 2 x 2 x 2 blocks: at most 8 per cube
}

int rb_rowgroups_bin(const double* node, int64_t nn, double x0, double y0, double z0, double h, int32_t nbx,
                     int32_t nby, int32_t nbz, int32_t* rows, int64_t* ng_out, void* work, size_t work_bytes,
                     void* stream) {
  if (!node || !rows || !ng_out || !work || nn < 1) return fail(RB_EARG, "rb_rowgroups_bin: bad arguments");
  if (!(h > 0) || !std::isfinite(h) || nbx < 1 || nby < 1 || nbz < 1)
    return fail(RB_EARG, "rb_rowgroups_bin: bad cube grid");
  // cube slots: 8 per 2 x 2 x 2 block of cubes (see rg_bin_kernel)
  const int64_t nb = 8 * (int64_t)((nbx + 1) / 2) * ((nby + 1) / 2) * ((nbz + 1) / 2);
  if (nb > (int64_t(1) << 26) || nn > INT32_MAX / kRGRows) return fail(RB_ESIZE, "rb_rowgroups_bin: grid too large");
  if (work_bytes < rb_rowgroups_work_bytes(nn, (int64_t)nbx * nby * nbz))
    return fail(RB_EARG, "rb_rowgroups_bin: workspace too small");
  cudaStream_t st = as_stream(stream);
  RgWork w;
  rg_carve(reinterpret_cast<char*>(work), nn, nb, &w);
  const unsigned gn = (unsigned)std::min<int64_t>(ceil_div(nn, 256), 148 * 16);
  const unsigned gb = (unsigned)std::min<int64_t>(ceil_div(nb, 256), 148 * 16);
  RB_CUDA_TRY(cudaMemsetAsync(w.cnt, 0, 4 * nb, st));
  RB_CUDA_TRY(cudaMemsetAsync(w.fill, 0, 4 * nb, st));
  rg_bin_kernel<<<gn, 256, 0, st>>>(nn, node, x0, y0, z0, 1.0 / h, nbx, nby, nbz, w.key, w.cnt);
  RB_LAUNCH_CHECK();
  rg_gcount_kernel<<<gb, 256, 0, st>>>(nb, w.cnt, w.gcnt);
  RB_LAUNCH_CHECK();
  RB_TRY(scan_exclusive(w.cnt, w.start, nb, w.scan, w.scan_bytes, st));
  RB_TRY(scan_exclusive(w.gcnt, w.gofs, nb, w.scan, w.scan_bytes, st));
  int32_t ng = 0;
  RB_CUDA_TRY(cudaMemcpyAsync(&ng, w.gofs + nb, 4, cudaMemcpyDeviceToHost, st));
  RB_CUDA_TRY(cudaStreamSynchronize(st));
  // every group slot starts empty (-1); short last groups of a cube keep it
  RB_CUDA_TRY(cudaMemsetAsync(rows, 0xff, (size_t)ng * kRGRows * 4, st));
  rg_scatter_kernel<<<gn, 256, 0, st>>>(nn, w.key, w.start, w.fill, w.tmp);
  RB_LAUNCH_CHECK();
  rg_place_kernel<<<(unsigned)std::min<int64_t>(ceil_div(nb, 8), 148 * 64), 256, 0, st>>>(nb, w.start, w.gofs,
                                                                                             w.tmp, rows);
  RB_LAUNCH_CHECK();
  *ng_out = ng;
  return RB_OK;
}

size_t rb_rowgroups_union_work_bytes(int64_t ng) {
  if (ng < 1) return 0;
  return (size_t)(ng + 1) * 4 + 256 + scan_work_bytes(ng);
}

int rb_rowgroups_union_count(const rb_csr* A, const int32_t* rows, int64_t ng, int32_t* uptr, int64_t* nu_out,
                             void* work, size_t work_bytes, void* stream) {
  if (!A || !rows || !uptr || !nu_out || !work || ng < 1) return fail(RB_EARG, "rb_rowgroups_union_count: bad arguments");
  if (work_bytes < rb_rowgroups_union_work_bytes(ng))
    return fail(RB_EARG, "rb_rowgroups_union_count: workspace too small");
  cudaStream_t st = as_stream(stream);
  int32_t* cnt = reinterpret_cast<int32_t*>(work);
  char* scan = reinterpret_cast<char*>(work) + ((size_t)(ng + 1) * 4 + 255) / 256 * 256;
  const unsigned grid = (unsigned)std::min<int64_t>(ceil_div(ng, 128), 148 * 32);
  rg_union_kernel<false><<<grid, 128, 0, st>>>(ng, rows, A->indptr, A->indices, cnt, nullptr, nullptr);
  RB_LAUNCH_CHECK();
  RB_TRY(scan_exclusive(cnt, uptr, ng, scan, scan_work_bytes(ng), st));
  int32_t nu = 0;
  RB_CUDA_TRY(cudaMemcpyAsync(&nu, uptr + ng, 4, cudaMemcpyDeviceToHost, st));
  RB_CUDA_TRY(cudaStreamSynchronize(st));
  *nu_out = nu;
  return RB_OK;
}

int rb_rowgroups_union_fill(const rb_csr* A, const int32_t* rows, int64_t ng, const int32_t* uptr, int32_t* ucol,
                            uint8_t* umask, void* stream) {
  if (!A || !rows || !uptr || !ucol || !umask || ng < 1) return fail(RB_EARG, "rb_rowgroups_union_fill: bad arguments");
  cudaStream_t st = as_stream(stream);
  const unsigned grid = (unsigned)std::min<int64_t>(ceil_div(ng, 128), 148 * 32);
  rg_union_kernel<true><<<grid, 128, 0, st>>>(ng, rows, A->indptr, A->indices, const_cast<int32_t*>(uptr), ucol,
                                              umask);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

}  // extern "C"
