// Aggregates of the two-level Krylov preconditioner: mesh nodes binned on a
// regular grid of cubes of edge h.  Every step is order-independent or runs
// in row order, so the result (aggregate numbering and the row lists) is the
// same on every run:
//   1. bin of every node, node count per bin (atomics: counts only);
//   2. nonempty bins numbered in bin order (scan of 0/1 flags) = aggregates,
//      agg_ptr = scan of the bin counts at the nonempty bins;
//   3. the rows of each aggregate in ascending order: per chunk of kChunk
//      consecutive rows the count of each aggregate, chunk offsets in chunk
//      order, then one warp per chunk places its rows 32 at a time, ranking
//      equal aggregates inside a step with __match_any_sync.
#include <algorithm>
#include <cmath>

#include "rb_common.cuh"

namespace rb {

constexpr int kAggMax = 4096;  // largest aggregate count (the coarse solver's limit)
constexpr int kChunk = 4096;   // rows per chunk of the ordered placement

__global__ void bin_kernel(int64_t nn, const double* __restrict__ node, double x0, double y0, double z0, double ih,
                           int32_t nbx, int32_t nby, int32_t nbz, int32_t* __restrict__ key,
                           int32_t* __restrict__ bincnt) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x) {
    const double* p = node + 3 * i;
    // NaN coordinates land in bin 0 (the clamps below see a false compare)
    int bx = (int)fmin(fmax(floor((p[0] - x0) * ih), 0.0), (double)(nbx - 1));
    int by = (int)fmin(fmax(floor((p[1] - y0) * ih), 0.0), (double)(nby - 1));
    int bz = (int)fmin(fmax(floor((p[2] - z0) * ih), 0.0), (double)(nbz - 1));
    bx = max(bx, 0);
    by = max(by, 0);
    bz = max(bz, 0);
    const int32_t b = bx + nbx * (by + nby * bz);
    key[i] = b;
    atomicAdd(bincnt + b, 1);
  }
}

__global__ void flag_kernel(int64_t nb, const int32_t* __restrict__ bincnt, int32_t* __restrict__ flag) {
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < nb; b += (int64_t)gridDim.x * blockDim.x)
    flag[b] = bincnt[b] > 0;
}

// agg_ptr[a] for the nonempty bins (binid -> a = binagg[b]); agg_ptr[nc] = nn
__global__ void aggptr_kernel(int64_t nb, int64_t nn, const int32_t* __restrict__ bincnt,
                              const int32_t* __restrict__ binagg, const int32_t* __restrict__ binstart,
                              int32_t* __restrict__ agg_ptr) {
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < nb; b += (int64_t)gridDim.x * blockDim.x) {
    if (bincnt[b] > 0) agg_ptr[binagg[b]] = binstart[b];
    if (b == nb - 1) agg_ptr[binagg[nb]] = (int32_t)nn;
  }
}

// agg of every row; per-chunk aggregate counts ccnt[chunk][a]
__global__ void chunk_count_kernel(int64_t nn, int64_t nc, const int32_t* __restrict__ key,
                                   const int32_t* __restrict__ binagg, int32_t* __restrict__ agg,
                                   int32_t* __restrict__ ccnt) {
  __shared__ int32_t cnt[kAggMax];
  for (int a = threadIdx.x; a < nc; a += blockDim.x) cnt[a] = 0;
  __syncthreads();
  const int64_t r0 = (int64_t)blockIdx.x * kChunk;
  const int64_t r1 = std::min<int64_t>(r0 + kChunk, nn);
  for (int64_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
    const int32_t a = binagg[key[i]];
    agg[i] = a;
    atomicAdd(cnt + a, 1);
  }
  __syncthreads();
  for (int a = threadIdx.x; a < nc; a += blockDim.x) ccnt[(int64_t)blockIdx.x * nc + a] = cnt[a];
}

// coff[chunk][a] = agg_ptr[a] + sum of ccnt[c][a] over the chunks c before
__global__ void chunk_offset_kernel(int64_t nchunk, int64_t nc, const int32_t* __restrict__ agg_ptr,
                                    const int32_t* __restrict__ ccnt, int32_t* __restrict__ coff) {
  for (int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; a < nc; a += (int64_t)gridDim.x * blockDim.x) {
    int32_t s = agg_ptr[a];
    for (int64_t c = 0; c < nchunk; ++c) {
      coff[c * nc + a] = s;
      s += ccnt[c * nc + a];
    }
  }
}

// one warp per chunk: rows in ascending order, 32 per step
__global__ void __launch_bounds__(32) place_kernel(int64_t nn, int64_t nc, const int32_t* __restrict__ agg,
                                                   const int32_t* __restrict__ coff, int32_t* __restrict__ agg_rows) {
  __shared__ int32_t pos[kAggMax];
  const int lane = threadIdx.x;
  for (int a = lane; a < nc; a += 32) pos[a] = coff[(int64_t)blockIdx.x * nc + a];
  __syncwarp();
  const int64_t r0 = (int64_t)blockIdx.x * kChunk;
  const int64_t r1 = std::min<int64_t>(r0 + kChunk, nn);
  const unsigned lt = (1u << lane) - 1u;
  for (int64_t s = r0; s < r1; s += 32) {
    const int64_t i = s + lane;
    const bool in = i < r1;
    const int32_t a = in ? agg[i] : -1 - lane;  // rows past the end match nobody
    const unsigned peers = __match_any_sync(0xffffffffu, a);
    if (in) agg_rows[pos[a] + __popc(peers & lt)] = (int32_t)i;
    __syncwarp();
    // the highest lane of each group advances that aggregate's cursor
    if (in && (peers >> lane) == 1u) pos[a] += __popc(peers);
    __syncwarp();
  }
}

struct AggWork {
  int32_t *key, *bincnt, *flag, *binagg, *binstart, *ccnt, *coff;
  char* scan;
  size_t scan_bytes;
};

static size_t agg_carve(char* base, int64_t nn, int64_t nbins, AggWork* w) {
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* p = base ? base + off : nullptr;
    off += (bytes + 255) / 256 * 256;
    return p;
  };
  const int64_t nchunk = ceil_div(nn, kChunk);
  AggWork t;
  t.key = (int32_t*)take(4 * nn);
  t.bincnt = (int32_t*)take(4 * nbins);
  t.flag = (int32_t*)take(4 * nbins);
  t.binagg = (int32_t*)take(4 * (nbins + 1));
  t.binstart = (int32_t*)take(4 * (nbins + 1));
  t.ccnt = (int32_t*)take(4 * (size_t)nchunk * kAggMax);
  t.coff = (int32_t*)take(4 * (size_t)nchunk * kAggMax);
  t.scan_bytes = scan_work_bytes(nbins);
  t.scan = take(t.scan_bytes);
  if (w) *w = t;
  return off;
}

}  // namespace rb

using namespace rb;

extern "C" {

size_t rb_coarse_aggregate_work_bytes(int64_t nn, int64_t nbins) {
  if (nn < 1 || nbins < 1) return 0;
  return agg_carve(nullptr, nn, nbins, nullptr);
}

int rb_coarse_aggregate(const double* node, int64_t nn, double x0, double y0, double z0, double h, int32_t nbx,
                        int32_t nby, int32_t nbz, int32_t* agg, int32_t* agg_ptr, int32_t* agg_rows, int64_t* nc_out,
                        void* work, size_t work_bytes, void* stream) {
  if (!node || !agg || !agg_ptr || !agg_rows || !nc_out || !work || nn < 1)
    return fail(RB_EARG, "rb_coarse_aggregate: bad arguments");
  if (!(h > 0) || !std::isfinite(h) || nbx < 1 || nby < 1 || nbz < 1)
    return fail(RB_EARG, "rb_coarse_aggregate: bad bin grid");
  const int64_t nbins = (int64_t)nbx * nby * nbz;
  if (nbins > (1 << 24) || nn > INT32_MAX - 1) return fail(RB_ESIZE, "rb_coarse_aggregate: bin grid too large");
  if (work_bytes < rb_coarse_aggregate_work_bytes(nn, nbins))
    return fail(RB_EARG, "rb_coarse_aggregate: workspace too small");
  cudaStream_t st = as_stream(stream);
  AggWork w;
  agg_carve(reinterpret_cast<char*>(work), nn, nbins, &w);
  const unsigned gn = (unsigned)std::min<int64_t>(ceil_div(nn, 256), 148 * 16);
  const unsigned gb = (unsigned)std::min<int64_t>(ceil_div(nbins, 256), 148 * 16);
  RB_CUDA_TRY(cudaMemsetAsync(w.bincnt, 0, 4 * nbins, st));
  bin_kernel<<<gn, 256, 0, st>>>(nn, node, x0, y0, z0, 1.0 / h, nbx, nby, nbz, w.key, w.bincnt);
  RB_LAUNCH_CHECK();
  flag_kernel<<<gb, 256, 0, st>>>(nbins, w.bincnt, w.flag);
  RB_LAUNCH_CHECK();
  RB_TRY(scan_exclusive(w.flag, w.binagg, nbins, w.scan, w.scan_bytes, st));
  RB_TRY(scan_exclusive(w.bincnt, w.binstart, nbins, w.scan, w.scan_bytes, st));
  int32_t nc = 0;
  RB_CUDA_TRY(cudaMemcpyAsync(&nc, w.binagg + nbins, 4, cudaMemcpyDeviceToHost, st));
  RB_CUDA_TRY(cudaStreamSynchronize(st));
  *nc_out = nc;
  if (nc > kAggMax) return fail(RB_ESIZE, "rb_coarse_aggregate: %d nonempty bins (at most %d)", nc, kAggMax);
  aggptr_kernel<<<gb, 256, 0, st>>>(nbins, nn, w.bincnt, w.binagg, w.binstart, agg_ptr);
  RB_LAUNCH_CHECK();
  const int64_t nchunk = ceil_div(nn, kChunk);
  chunk_count_kernel<<<(unsigned)nchunk, 256, 0, st>>>(nn, nc, w.key, w.binagg, agg, w.ccnt);
  RB_LAUNCH_CHECK();
  chunk_offset_kernel<<<(unsigned)ceil_div(nc, 128), 128, 0, st>>>(nchunk, nc, agg_ptr, w.ccnt, w.coff);
  RB_LAUNCH_CHECK();
  place_kernel<<<(unsigned)nchunk, 32, 0, st>>>(nn, nc, agg, w.coff, agg_rows);
  RB_LAUNCH_CHECK();
  return RB_OK;
}

}  // extern "C"
