// Gram matrix H = alpha * J J^T of the Gauss-Newton step on the 5th-generation
// tensor cores (tcgen05, TF32 inputs, FP32 accumulation in tensor memory).
//
// J is M x K FP32, row-major (K contiguous): the Jacobian rows of redbirdpy's
// jac / matreform layout.  Both MMA operands are row blocks of the same J and
// are "K-major", so one TMA tensor map (box 32 x 128, 128-byte swizzle)
// serves every load.  A CTA computes a 256 x 256 tile of H (over one K
// range at a time) as two M = 128, N = 256 MMAs that share the B operand
// (two accumulators filling all 512 TMEM columns), which halves the operand
// bytes per FLOP against a single 128 x 256 tile.  Only tiles on or above the
// diagonal are computed; a second kernel mirrors the upper triangle into the
// lower one.  One persistent CTA per SM claims (tile, K range) items in turn
// (see gram_tf32_kernel), and rows longer than 1 MB are read from compact
// copies of one 65536-column slab at a time (gram_run).
//
// Warp roles (192 threads): warp 0 = TMA producer (one lane), warp 1 = TMEM
// allocator + MMA issuer (one lane), warps 2..5 = epilogue (each reads the
// 32 TMEM lanes of its quarter with tcgen05.ld and writes FP64 rows of H).
// A 3-stage shared-memory ring (64 KB per stage) is synchronised with
// mbarriers; every wait is bounded and reports a timeout through an error
// word instead of hanging.
#include <cuda.h>

#include <algorithm>

#include "rb_common.cuh"
#include "rb_tc.cuh"

namespace rb {

constexpr int kGM = 256;   // tile rows (A, two MMA halves of 128)
constexpr int kGMH = 128;  // rows per MMA / per TMA box
constexpr int kGN = 256;   // tile columns (B rows)
constexpr int kGK = 32;    // FP32 elements per 128-byte row of a stage (64 for BF16)
constexpr int kGStages = 3;
constexpr int kGABytes = kGM * kGK * 4;  // 32 KB
constexpr int kGBBytes = kGN * kGK * 4;  // 32 KB
constexpr int kGBoxBytes = kGMH * kGK * 4;  // 16 KB
constexpr int kGStageBytes = kGABytes + kGBBytes;
constexpr int kGSmem = kGStages * kGStageBytes + 1024 + 256;  // ring + alignment + barriers
constexpr int kGThreads = 192;
constexpr uint32_t kGTmemCols = 512;  // two 128 x 256 FP32 accumulators (rows 0-127, 128-255)
// K-blocks per accumulation chunk: the tensor cores' FP32 accumulator is
// drained into the FP64 output every chunk * 32 K-elements, because its
// rounding error grows linearly with the chunk length (measured ~2e-5
// relative per 4096 K; ~8e-3 after one undrained sweep of K = 10^6).  The
// split form (tf32x3) drains every 4096 K; the plain TF32 form every 16384 K
// (~1e-4, below what its rounded inputs allow), so that its MMAs wait on
// four times fewer drains.
constexpr int kGItems = 4;  // item indices the producer may claim ahead of the epilogue
constexpr int kGChunk = 128;
constexpr int kGChunkTf32 = 512;
constexpr int kGChunkBf16 = 256;  // the same 16384 K with 64 BF16 elements per K-block
constexpr long long kGWaitLimit = kTcWaitLimit;  // polls before a wait gives up (seconds)

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
      : "memory");
}

// instruction descriptor: D = F32, both operands K-major, M = 128, N = 256;
// A = B = TF32 (kind::tf32, format 2) or A = B = BF16 (kind::f16, format 1)
constexpr uint32_t kGIdesc = umma_idesc(2, kGMH, kGN);
constexpr uint32_t kGIdescBf16 = umma_idesc(1, kGMH, kGN);

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
  umma_tf32_i(tmem_d, a, b, kGIdesc, accumulate);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
  umma_bf16_i(tmem_d, a, b, kGIdescBf16, accumulate);
}

// number of 128-row blocks of tile column bj that touch the upper triangle
__device__ __host__ __forceinline__ int64_t gram_col_tiles(int64_t bj, int64_t nbi) {
  const int64_t need = (bj * kGN + kGN - 1) / kGM + 1;
  return need < nbi ? need : nbi;
}

// tile t of the upper triangle -> its row offsets (i0 in H's rows, j0 in its
// columns): tiles are numbered down each tile column, column after column
__device__ __forceinline__ void gram_tile(int64_t t, int64_t nbi, int64_t nbj, int& i0, int& j0) {
  int64_t bj = 0;
  while (bj < nbj - 1 && t >= gram_col_tiles(bj, nbi)) t -= gram_col_tiles(bj++, nbi);
  i0 = (int)(t * kGM);
  j0 = (int)(bj * kGN);
}

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ bool aborted(const int* err) { return *(volatile const int*)err != 0; }

// Persistent form: one CTA per SM claims work items (tile t, K segment s of
// kspan) from a global counter in segment-major order, item = s * tiles + t,
// and hands each index to its MMA lane and epilogue warps through a small
// shared-memory ring.  Claiming instead of a fixed deal lets an SM that runs
// slower take fewer items (a fixed round-robin deal measured 270 ms against
// 223 ms at 8192 x 1,040,502), and short items leave a short last round
// (2112 items per launch instead of 528 tiles in 4 waves, the last one 57%
// full: 238 ms).  The FP64 partial sums of tile t for segment s are added to
// H only after those of segment s - 1: each epilogue warp publishes its rows
// with a fenced increment of done[t] and waits for done[t] >= 4 s before its
// first add.  Item i depends only on item i - tiles, claimed earlier, and all
// CTAs are resident (cooperative launch, one CTA per SM), so the waits always
// end; they are bounded all the same.  With nseg == 1 (one item per tile,
// used when the tile count outgrows the progress counters) nothing waits.
//
// BF16: J stored as BF16 (64 elements per 128-byte stage row), one pass
template <bool BF16>
__global__ void __launch_bounds__(kGThreads, 1)
gram_tf32_kernel(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ CUtensorMap tmap_lo, int segs,
                 int64_t M, int64_t kbeg, int64_t K, int64_t kspan, int64_t tiles, int accumulate,
                 double* __restrict__ H, int64_t ldh, double alpha, int* __restrict__ done,
                 unsigned long long* __restrict__ next, int* __restrict__ err) {
  // K range [kbeg, kbeg + K) of this launch in segments of kspan; accumulate:
  // add segment 0 to H instead of writing it
  extern __shared__ __align__(1024) unsigned char gsm_raw[];
  unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(gsm_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + kGStages * kGStageBytes);
  uint64_t* empty = full + kGStages;
  uint64_t* tfull = empty + kGStages;  // accumulators ready for the epilogue
  uint64_t* tempty = tfull + 1;        // accumulators drained by the epilogue
  uint64_t* mdone = tempty + 1;        // every MMA of this CTA complete (exit)
  uint64_t* ifull = mdone + 1;         // item ring: index written by the producer
  uint64_t* iempty = ifull + kGItems;  // item ring: read by the MMA lane and the 4 epilogue warps
  int64_t* sitem = reinterpret_cast<int64_t*>(iempty + kGItems);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sitem + kGItems);

  const int64_t nbi = (M + kGM - 1) / kGM, nbj = (M + kGN - 1) / kGN;
  const int64_t nseg = (K + kspan - 1) / kspan;
  const int64_t items = tiles * nseg;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kGStages; ++s) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), 1);
    }
    mbar_init(smem_u32(tfull), 1);
    mbar_init(smem_u32(tempty), 4 * 32);
    mbar_init(smem_u32(mdone), 1);
    for (int s = 0; s < kGItems; ++s) {
      mbar_init(smem_u32(&ifull[s]), 1);
      mbar_init(smem_u32(&iempty[s]), 1 + 4);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kGTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  // segs == 1: H = J J^T.  segs == 3 (split precision, J = hi + lo):
  // H = hi hi^T + hi lo^T + lo hi^T, one K sweep per product, one accumulator
  constexpr int kE = BF16 ? 2 * kGK : kGK;  // elements per 128-byte stage row
  const int chunk = BF16 ? kGChunkBf16 : (segs == 1) ? kGChunkTf32 : kGChunk;  // K-blocks between drains
  // K-blocks of one pass over segment s
  auto seg_blocks = [&](int64_t s) -> int {
    const int64_t k0 = s * kspan, k1 = (k0 + kspan < K) ? k0 + kspan : K;
    return (int)((k1 - k0 + kE - 1) / kE);
  };

  if (warp == 0) {
    if (lane == 0) {
      uint32_t g = 0;  // stages issued by this CTA
      bool ok = true;
      for (uint32_t n = 0; ok; ++n) {
        // claim the next item and hand its index to the other roles
        const int slot = (int)(n % kGItems);
        if (n >= (uint32_t)kGItems && !mbar_wait(smem_u32(&iempty[slot]), ((n / kGItems) - 1) & 1, err, 8)) break;
        const int64_t item = aborted(err) ? items : (int64_t)atomicAdd(next, 1ull);
        sitem[slot] = item < items ? item : items;
        mbar_arrive(smem_u32(&ifull[slot]));
        if (item >= items) break;
        const int64_t s = item / tiles;
        int i0, j0;
        gram_tile(item - s * tiles, nbi, nbj, i0, j0);
        const int nk1 = seg_blocks(s), nk = nk1 * segs;
        for (int kb = 0; kb < nk; ++kb) {
          const int st = (int)(g % kGStages);
          if (g >= (uint32_t)kGStages && !mbar_wait(smem_u32(&empty[st]), ((g / kGStages) - 1) & 1, err, 1)) {
            ok = false;
            break;
          }
          const uint32_t a = smem_u32(sm + st * kGStageBytes);
          const uint32_t b = a + kGABytes;
          const uint32_t bar = smem_u32(&full[st]);
          const int seg = kb / nk1;
          const int kx = (int)(kbeg + s * kspan) + (kb - seg * nk1) * kE;
          const CUtensorMap* ma = (seg == 2) ? &tmap_lo : &tmap;
          const CUtensorMap* mb = (seg == 1) ? &tmap_lo : &tmap;
          mbar_expect_tx(bar, kGStageBytes);
          tma_load_2d(a, ma, bar, kx, i0);
          tma_load_2d(a + kGBoxBytes, ma, bar, kx, i0 + kGMH);
          tma_load_2d(b, mb, bar, kx, j0);
          tma_load_2d(b + kGBoxBytes, mb, bar, kx, j0 + kGMH);
          ++g;
        }
      }
      // the copies still in flight land before the CTA exits
      for (uint32_t h = g > (uint32_t)kGStages ? g - kGStages : 0u; h < g; ++h)
        mbar_wait(smem_u32(&full[h % kGStages]), (h / kGStages) & 1, err, 5);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      uint32_t g = 0, cc = 0;  // stages consumed, accumulator chunks committed
      bool ok = true;
      for (uint32_t n = 0; ok; ++n) {
        const int slot = (int)(n % kGItems);
        if (!mbar_wait(smem_u32(&ifull[slot]), (n / kGItems) & 1, err, 9)) break;
        const int64_t item = sitem[slot];
        mbar_arrive(smem_u32(&iempty[slot]));
        if (item >= items) break;
        const int nk = seg_blocks(item / tiles) * segs;
        for (int kb = 0; kb < nk; ++kb) {
          const int st = (int)(g % kGStages);
          const bool first = (kb % chunk) == 0;
          const bool last = (kb % chunk) == chunk - 1 || kb == nk - 1;
          // a new chunk waits until the epilogue drained the previous one
          if (first && cc >= 1 && !mbar_wait(smem_u32(tempty), (cc - 1) & 1, err, 4)) {
            ok = false;
            break;
          }
          if (!mbar_wait(smem_u32(&full[st]), (g / kGStages) & 1, err, 2)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t a = smem_u32(sm + st * kGStageBytes);
          const uint32_t b = a + kGABytes;
#pragma unroll
          for (int k = 0; k < 4; ++k) {  // 32 bytes of K per MMA: 8 TF32 or 16 BF16 elements
            const uint64_t bd = umma_desc_sw128(b + 32 * k);
            const uint32_t acc = !(first && k == 0);
            if constexpr (BF16) {
              umma_bf16(tmem, umma_desc_sw128(a + 32 * k), bd, acc);
              umma_bf16(tmem + kGN, umma_desc_sw128(a + kGBoxBytes + 32 * k), bd, acc);
            } else {
              umma_tf32(tmem, umma_desc_sw128(a + 32 * k), bd, acc);
              umma_tf32(tmem + kGN, umma_desc_sw128(a + kGBoxBytes + 32 * k), bd, acc);
            }
          }
          umma_commit(smem_u32(&empty[st]));
          if (last) {
            umma_commit(smem_u32(tfull));
            ++cc;
          }
          ++g;
        }
      }
      // every MMA issued completes before the accumulators are freed
      umma_commit(smem_u32(mdone));
      mbar_wait(smem_u32(mdone), 0, err, 6);
    }
  } else {
    // epilogue: warp w reads TMEM lanes 32*(w%4) .. +31 of both accumulators
    // (tile rows r and r + 128) and adds each chunk's FP32 partial sums into
    // the FP64 output rows
    const int q = warp & 3;
    const int row = 32 * q + lane;
    uint32_t cc = 0;  // accumulator chunks drained
    bool ok = true;
    for (uint32_t n = 0; ok; ++n) {
      const int slot = (int)(n % kGItems);
      int64_t item = items;
      if (lane == 0) {
        if (mbar_wait(smem_u32(&ifull[slot]), (n / kGItems) & 1, err, 10)) {
          item = sitem[slot];
          mbar_arrive(smem_u32(&iempty[slot]));
        }
      }
      item = __shfl_sync(0xffffffffu, item, 0);
      if (item >= items) break;
      const int64_t s = item / tiles, t = item - s * tiles;
      int i0, j0;
      gram_tile(t, nbi, nbj, i0, j0);
      const int nk = seg_blocks(s) * segs;
      const int nchunk = (nk + chunk - 1) / chunk;
      if (s > 0) {
        // the four epilogue warps of segment s - 1 have added their rows
        bool seen = true;
        if (lane == 0) {
          const int want = 4 * (int)s;
          long long i = 0;
          // stop at once when another role has already failed (its error code stays)
          while (ld_acquire(done + t) < want && !aborted(err) && ++i < kGWaitLimit) __nanosleep(64);
          seen = ld_acquire(done + t) >= want;
          if (!seen && i >= kGWaitLimit) atomicExch(err, 7);
        }
        if (!__shfl_sync(0xffffffffu, (int)seen, 0)) break;
        (void)ld_acquire(done + t);  // every lane orders its reads of H after the flag
      }
      for (int c = 0; c < nchunk; ++c, ++cc) {
        // warp-uniform outcome: tcgen05.ld below needs the whole warp
        const bool got = __all_sync(0xffffffffu, mbar_wait(smem_u32(tfull), cc & 1, err, 3));
        if (!got) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const bool write = (c == 0 && s == 0 && !accumulate);
#pragma unroll 1
        for (int h = 0; h < 2; ++h) {
          const int64_t gi = (int64_t)i0 + h * kGMH + row;
#pragma unroll 1
          for (int c0 = 0; c0 < kGN; c0 += 32) {
            uint32_t v[32];
            const uint32_t taddr = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(h * kGN + c0);
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                  "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                  "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (gi < M) {
              double* dst = H + gi * ldh + j0 + c0;
#pragma unroll
              for (int u = 0; u < 32; ++u)
                if ((int64_t)j0 + c0 + u < M) {
                  const double x = alpha * (double)__uint_as_float(v[u]);
                  dst[u] = write ? x : dst[u] + x;
                }
            }
          }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(tempty)) : "memory");
      }
      if (!ok) break;
      if (nseg > 1) {
        // publish this warp's rows of tile t through segment s
        __threadfence();
        __syncwarp();
        if (lane == 0) {
          __threadfence();
          atomicAdd(done + t, 1);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kGTmemCols));
}

// S[r][0 .. nb) = J[r][b0 .. b0 + nb) in bytes (16-byte pieces, nb a multiple
// of 16): the column slab of one launch, copied into a compact buffer; rows
// on grid y, 16-byte pieces of a row on grid x, four per thread in flight
__global__ void __launch_bounds__(256) slab_copy_kernel(const unsigned char* __restrict__ J, int64_t ldj_b, int64_t b0,
                                                        int64_t nb, unsigned char* __restrict__ S, int64_t lds_b,
                                                        int64_t M) {
  const int64_t per_row = nb >> 4;
  const int64_t step = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = blockIdx.y; r < M; r += gridDim.y) {
    const int4* __restrict__ src = reinterpret_cast<const int4*>(J + r * ldj_b + b0);
    int4* __restrict__ dst = reinterpret_cast<int4*>(S + r * lds_b);
    int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    for (; c + 3 * step < per_row; c += 4 * step) {
      const int4 v0 = __ldcs(src + c), v1 = __ldcs(src + c + step), v2 = __ldcs(src + c + 2 * step),
                 v3 = __ldcs(src + c + 3 * step);
      dst[c] = v0;
      dst[c + step] = v1;
      dst[c + 2 * step] = v2;
      dst[c + 3 * step] = v3;
    }
    for (; c < per_row; c += step) dst[c] = __ldcs(src + c);
  }
}

// H[j][i] = H[i][j] for i < j (upper triangle -> lower)
__global__ void mirror_upper_kernel(double* __restrict__ H, int64_t M, int64_t ldh) {
  __shared__ double tile[32][33];
  const int64_t bi = blockIdx.y, bj = blockIdx.x;
  if (bj < bi) return;  // tiles of the upper triangle only
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int r = ty; r < 32; r += blockDim.y) {
    const int64_t i = bi * 32 + r, j = bj * 32 + tx;
    tile[r][tx] = (i < M && j < M) ? H[i * ldh + j] : 0.0;
  }
  __syncthreads();
  for (int r = ty; r < 32; r += blockDim.y) {
    const int64_t i = bj * 32 + r, j = bi * 32 + tx;  // destination row i (lower part)
    if (i < M && j < M && i > j) H[i * ldh + j] = tile[tx][r];
  }
}

typedef decltype(&cuTensorMapEncodeTiled) EncodeTiledFn;

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

}  // namespace rb

using namespace rb;

static int make_map(CUtensorMap* map, const void* J, int64_t M, int64_t K, int64_t ldj, bool bf16 = false) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return fail(RB_ECUDA, "rb_gram: cuTensorMapEncodeTiled unavailable");
  cuuint64_t gdim[2] = {(cuuint64_t)K, (cuuint64_t)M};
  cuuint64_t gstride[1] = {(cuuint64_t)ldj * (bf16 ? 2 : 4)};
  cuuint32_t box[2] = {(cuuint32_t)(bf16 ? 2 * kGK : kGK), (cuuint32_t)kGMH};
  cuuint32_t estride[2] = {1, 1};
  CUresult r = enc(map, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                   const_cast<void*>(J), gdim, gstride, box, estride,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(RB_ECUDA, "rb_gram: cuTensorMapEncodeTiled failed (%d)", (int)r);
  return RB_OK;
}

extern "C" {

// workspace: the error word, the item counter (byte 128), then one progress
// counter per tile from byte 256, for up to kGFlags tiles (M up to about
// 92,000 rows); larger M takes whole tiles as items, which needs no counters
constexpr int64_t kGFlags = 65536;
size_t rb_gram_work_bytes(void) { return 256 + (size_t)kGFlags * sizeof(int); }

// K per launch: a launch boundary brings every CTA back to the same K, so the
// slab of J they share stays in L2 (one launch over all of K let the CTAs
// drift apart: 276 against 238 ms at 8192 x 1,040,502)
constexpr int64_t kGSeg = 65536;
// rows longer than this (bytes) are staged slab by slab when a buffer is given
constexpr int64_t kGStageRow = 1 << 20;

size_t rb_gram_stage_bytes(int64_t M, int64_t K, int64_t ldj, int32_t elem_bytes, int32_t split) {
  if (M < 1 || K < 1 || (elem_bytes != 2 && elem_bytes != 4) || ldj * elem_bytes <= kGStageRow) return 0;
  return (size_t)M * kGSeg * elem_bytes * (split ? 2 : 1) + 256;
}

static int gram_run(const void* J, const void* Jlo, bool bf16, int64_t M, int64_t K, int64_t ldj, double alpha,
                    double* H, int64_t ldh, void* stage, size_t stage_bytes, void* work, size_t work_bytes,
                    void* stream) {
  if (!J || !H || !work || M < 1 || K < 1 || ldj < K || ldh < M)
    return fail(RB_EARG, "rb_gram: bad arguments");
  if (work_bytes < rb_gram_work_bytes()) return fail(RB_EARG, "rb_gram: workspace too small");
  const int64_t lda = bf16 ? 8 : 4;  // elements per 16 bytes
  if ((reinterpret_cast<uintptr_t>(J) & 15) || (Jlo && (reinterpret_cast<uintptr_t>(Jlo) & 15)) || (ldj % lda))
    return fail(RB_EARG, "rb_gram: J must be 16-byte aligned with a row stride that is a multiple of 16 bytes");
  if (M > (int64_t)1 << 30 || K > (int64_t)1 << 30) return fail(RB_ESIZE, "rb_gram: matrix too large");
  const int eb = bf16 ? 2 : 4;
  const size_t need = rb_gram_stage_bytes(M, K, ldj, eb, Jlo != nullptr);
  const bool staged = stage && need > 0;
  if (staged && (stage_bytes < need || (reinterpret_cast<uintptr_t>(stage) & 15)))
    return fail(RB_EARG, "rb_gram: staging buffer too small or not 16-byte aligned");
  unsigned char* S = static_cast<unsigned char*>(stage);
  unsigned char* Slo = staged && Jlo ? S + (size_t)M * kGSeg * eb : nullptr;
  CUtensorMap map, map_lo;
  if (!staged) {
    RB_TRY(make_map(&map, J, M, K, ldj, bf16));
    RB_TRY(make_map(&map_lo, Jlo ? Jlo : J, M, K, ldj, bf16));
  }
  int segs = Jlo ? 3 : 1;
  cudaStream_t st = as_stream(stream);
  int* err = reinterpret_cast<int*>(work);
  unsigned long long* next = reinterpret_cast<unsigned long long*>(static_cast<unsigned char*>(work) + 128);
  int* done = reinterpret_cast<int*>(static_cast<unsigned char*>(work) + 256);
  RB_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), st));
  const int64_t nbi = ceil_div(M, kGM), nbj = ceil_div(M, kGN);
  int64_t tiles = 0;
  for (int64_t bj = 0; bj < nbj; ++bj) tiles += gram_col_tiles(bj, nbi);
  const void* fn = bf16 ? reinterpret_cast<const void*>(&gram_tf32_kernel<true>)
                        : reinterpret_cast<const void*>(&gram_tf32_kernel<false>);
  RB_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kGSmem));
  int dev = 0, sms = 0, per_sm = 0;
  RB_CUDA_TRY(cudaGetDevice(&dev));
  RB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  RB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kGThreads, kGSmem));
  if (per_sm < 1 || sms < 1) return fail(RB_ECUDA, "rb_gram: the tile kernel does not fit on an SM");
  const int64_t resident = (int64_t)sms * per_sm;
  // Inside a launch the items are (tile, 16384 K) pairs, one accumulator
  // chunk of the single-pass forms, so the last round is short: 2112 items on
  // 148 SMs instead of 528 tiles in 4 waves with the last one 57% full.
  const int64_t kseg = kGSeg, kitem = 16384;  // multiples of every stage row
  int64_t kspan = kitem, kbeg = 0, klen = 0, koff = 0;
  int accumulate = 0;
  // staged: copy the launch's slab of J (and Jlo) into the compact buffer and
  // map that instead; the kernel's K offset is then 0
  auto stage_slab = [&]() -> int {
    if (!staged) {
      koff = kbeg;
      return RB_OK;
    }
    const int64_t nb = (klen * eb + 15) / 16 * 16;
    const dim3 g((unsigned)std::max<int64_t>(1, ceil_div(nb / 16, 256 * 4)), (unsigned)std::min<int64_t>(M, 65535));
    slab_copy_kernel<<<g, 256, 0, st>>>(static_cast<const unsigned char*>(J), ldj * eb, kbeg * eb, nb, S, kseg * eb, M);
    RB_LAUNCH_CHECK();
    if (Jlo) {
      slab_copy_kernel<<<g, 256, 0, st>>>(static_cast<const unsigned char*>(Jlo), ldj * eb, kbeg * eb, nb, Slo,
                                          kseg * eb, M);
      RB_LAUNCH_CHECK();
    }
    RB_TRY(make_map(&map, S, M, klen, kseg, bf16));
    RB_TRY(make_map(&map_lo, Jlo ? Slo : S, M, klen, kseg, bf16));
    koff = 0;
    return RB_OK;
  };
  if (tiles <= kGFlags) {
    for (kbeg = 0; kbeg < K; kbeg += kseg) {
      klen = std::min<int64_t>(kseg, K - kbeg);
      accumulate = kbeg > 0;
      RB_TRY(stage_slab());
      RB_CUDA_TRY(cudaMemsetAsync(next, 0, 128 + (size_t)tiles * sizeof(int), st));  // item counter, progress
      const int64_t items = tiles * ceil_div(klen, kspan);
      const dim3 grid((unsigned)std::min<int64_t>(items, resident)), block(kGThreads);
      void* args[] = {(void*)&map,  (void*)&map_lo, (void*)&segs,       (void*)&M,   (void*)&koff,
                      (void*)&klen, (void*)&kspan,  (void*)&tiles,      (void*)&accumulate, (void*)&H,
                      (void*)&ldh,  (void*)&alpha,  (void*)&done,       (void*)&next, (void*)&err};
      // cooperative: every CTA resident, so the per-tile ordering waits end
      RB_CUDA_TRY(cudaLaunchCooperativeKernel(fn, grid, block, args, (size_t)kGSmem, st));
    }
  } else {
    // more tiles than progress counters: items are whole tiles of one launch
    // (no ordering between CTAs needed)
    kspan = kseg;
    const dim3 grid((unsigned)std::min<int64_t>(tiles, resident));
    for (kbeg = 0; kbeg < K; kbeg += kseg) {
      klen = std::min<int64_t>(kseg, K - kbeg);
      accumulate = kbeg > 0;
      RB_TRY(stage_slab());
      RB_CUDA_TRY(cudaMemsetAsync(next, 0, sizeof(unsigned long long), st));
      if (bf16)
        gram_tf32_kernel<true><<<grid, kGThreads, kGSmem, st>>>(map, map_lo, 1, M, koff, klen, kspan, tiles,
                                                                 accumulate, H, ldh, alpha, done, next, err);
      else
        gram_tf32_kernel<false><<<grid, kGThreads, kGSmem, st>>>(map, map_lo, segs, M, koff, klen, kspan, tiles,
                                                                  accumulate, H, ldh, alpha, done, next, err);
      RB_LAUNCH_CHECK();
    }
  }
  dim3 mg((unsigned)ceil_div(M, 32), (unsigned)ceil_div(M, 32));
  mirror_upper_kernel<<<mg, dim3(32, 8), 0, st>>>(H, M, ldh);
  RB_LAUNCH_CHECK();
  int herr = 0;
  RB_CUDA_TRY(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  RB_CUDA_TRY(cudaStreamSynchronize(st));
  if (herr) return fail(RB_ECUDA, "rb_gram: pipeline wait timed out (stage %d)", herr);
  return RB_OK;
}

int rb_gram(const float* J, const float* Jlo, int64_t M, int64_t K, int64_t ldj, double alpha, double* H, int64_t ldh,
            void* work, size_t work_bytes, void* stream) {
  return gram_run(J, Jlo, false, M, K, ldj, alpha, H, ldh, nullptr, 0, work, work_bytes, stream);
}

int rb_gram_staged(const float* J, const float* Jlo, int64_t M, int64_t K, int64_t ldj, double alpha, double* H,
                   int64_t ldh, void* stage, size_t stage_bytes, void* work, size_t work_bytes, void* stream) {
  return gram_run(J, Jlo, false, M, K, ldj, alpha, H, ldh, stage, stage_bytes, work, work_bytes, stream);
}

int rb_gram_bf16(const void* J, int64_t M, int64_t K, int64_t ldj, double alpha, double* H, int64_t ldh, void* work,
                 size_t work_bytes, void* stream) {
  return gram_run(J, nullptr, true, M, K, ldj, alpha, H, ldh, nullptr, 0, work, work_bytes, stream);
}

int rb_gram_bf16_staged(const void* J, int64_t M, int64_t K, int64_t ldj, double alpha, double* H, int64_t ldh,
                        void* stage, size_t stage_bytes, void* work, size_t work_bytes, void* stream) {
  return gram_run(J, nullptr, true, M, K, ldj, alpha, H, ldh, stage, stage_bytes, work, work_bytes, stream);
}

}  // extern "C"
