// brt_sort.cu -- stable LSD "onesweep" radix sort of (key, value) pairs.
//
// Replaces the reference's 3-kernel-per-digit CUDA-SDK sort
// (PlugIns/EnvGrid3D/radixsort.cu:50-80, radixsort_kernel.cu:106-580) with a
// single kernel per digit pass written from the published onesweep method
// (Adinets & Merrill, "Onesweep: A Faster Least Significant Digit Radix Sort
// for GPUs", 2022):
//   * one global histogram of every pass's digits, computed up front;
//   * tiles are claimed in order through an atomic counter, ranked inside the
//     CTA with warp-level multisplit (match_any + popc; items are processed in
//     input order, so equal digits keep their order: the sort is stable);
//   * each tile publishes its per-digit count and finds its global offset by
//     decoupled look-back over its predecessors' published counts;
//   * the tile is reordered by digit in shared memory and written out, so
//     equal-digit runs leave as contiguous, coalesced stores.
// Every look-back wait is bounded: after the plan's spin limit of polls the
// tile records kDevErrLookback in the error word and continues, so a kernel
// never hangs the GPU (the host then reports BRT_ERR_TIMEOUT).  A tile that
// gives up takes a partial prefix: its outputs land at positions below the
// right ones, still inside [0, n), so a failed sort is wrong but never writes
// out of bounds.
#include "brt_internal.cuh"

#include <algorithm>
#include <string>

namespace brt {
namespace {

constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagInc = 2u << 30;
constexpr uint32_t kFlagMask = 3u << 30;
constexpr uint32_t kValMask = (1u << 30) - 1;

// Exclusive scan of one value per thread across the CTA; returns the
// exclusive prefix and writes the total to *total.
template <int THREADS>
__device__ __forceinline__ uint32_t blockExclusiveScan(uint32_t v, uint32_t* sWarpSums, uint32_t* total) {
  constexpr int WARPS = THREADS / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sWarpSums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < WARPS ? sWarpSums[lane] : 0u;
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < WARPS) sWarpSums[lane] = wi - w;  // exclusive warp offsets
    if (lane == WARPS - 1) sWarpSums[WARPS] = wi;
  }
  __syncthreads();
  uint32_t r = sWarpSums[warp] + x - v;
  *total = sWarpSums[WARPS];
  __syncthreads();
  return r;
}

template <int BITS>
__global__ void __launch_bounds__(kSortThreads)
onesweepKernel(const uint2* __restrict__ in, uint2* __restrict__ out, uint32_t n, uint32_t shift,
               uint32_t mask, const uint32_t* __restrict__ hist, uint32_t* __restrict__ status,
               uint32_t* __restrict__ counter, uint32_t* __restrict__ errWord, const uint32_t* gate,
               LookbackWait wait) {
  constexpr int BINS = 1 << BITS;
  constexpr int T = kSortThreads;
  constexpr int WARPS = T / 32;
  constexpr int IPT = (int)sortItemsFor(BITS);
  constexpr int TILE = (int)sortTileFor(BITS);
  constexpr int DPT = (BINS + T - 1) / T;  // digits per thread (consecutive)

  __shared__ uint32_t sWarp[WARPS][BINS];
  __shared__ uint32_t sDigitStart[BINS];
  __shared__ uint32_t sGlobal[BINS];
  __shared__ uint2 sItems[TILE];
  __shared__ uint32_t sScan[WARPS + 1];
  __shared__ uint32_t sTile;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (gate && *gate != kResortFullSort) return;  // this step's order came from the incremental re-sort
  if (tid == 0) sTile = atomicAdd(counter, 1u);
  for (int k = tid; k < WARPS * BINS; k += T) (&sWarp[0][0])[k] = 0u;
  __syncthreads();
  const uint32_t tile = sTile;
  const uint32_t tileBase = tile * (uint32_t)TILE;
  if (tileBase >= n) return;  // counters not reset: never index past the input

  // Warp-striped load: warp w owns the contiguous run [w*32*IPT, (w+1)*32*IPT).
  uint2 item[IPT];
  uint32_t dig[IPT];
  uint32_t off[IPT];
  const uint32_t wbase = tileBase + (uint32_t)warp * 32u * IPT;
#pragma unroll
  for (int i = 0; i < IPT; ++i) {
    uint32_t idx = wbase + (uint32_t)i * 32u + lane;
    if (idx < n) {
      item[i] = in[idx];
      dig[i] = (item[i].x >> shift) & mask;
    } else {
      item[i] = make_uint2(0u, 0u);
      dig[i] = BINS;  // sentinel: not counted, not written
    }
  }
  // Warp-level multisplit ranking, items in input order.
  const uint32_t ltmask = (1u << lane) - 1u;
#pragma unroll
  for (int i = 0; i < IPT; ++i) {
    const uint32_t d = dig[i];
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (lane == leader && d < (uint32_t)BINS) {
      base = sWarp[warp][d];
      sWarp[warp][d] = base + __popc(peers);
    }
    base = __shfl_sync(0xffffffffu, base, leader);
    off[i] = base + __popc(peers & ltmask);
    __syncwarp();
  }
  __syncthreads();

  // Per digit: exclusive prefix over warps and the tile total.
  uint32_t cnt[DPT];
#pragma unroll
  for (int k = 0; k < DPT; ++k) {
    const int d = tid * DPT + k;
    uint32_t run = 0;
    if (d < BINS) {
#pragma unroll
      for (int w = 0; w < WARPS; ++w) {
        uint32_t t = sWarp[w][d];
        sWarp[w][d] = run;
        run += t;
      }
      // Publish as early as possible so successors can proceed.
      stRelaxed(&status[(size_t)tile * BINS + d], (tile == 0 ? kFlagInc : kFlagAgg) | run);
    }
    cnt[k] = run;
  }
  // Tile-local digit starts and global digit starts.
  uint32_t sumCnt = 0, sumHist = 0;
  uint32_t hv[DPT];
#pragma unroll
  for (int k = 0; k < DPT; ++k) {
    const int d = tid * DPT + k;
    hv[k] = d < BINS ? __ldg(&hist[d]) : 0u;
    sumCnt += cnt[k];
    sumHist += hv[k];
  }
  uint32_t tot;
  uint32_t exclCnt = blockExclusiveScan<T>(sumCnt, sScan, &tot);
  uint32_t exclHist = blockExclusiveScan<T>(sumHist, sScan, &tot);

  // Decoupled look-back per digit.
#pragma unroll
  for (int k = 0; k < DPT; ++k) {
    const int d = tid * DPT + k;
    if (d < BINS) {
      uint32_t excl = 0;
      if (tile > 0) {
        int p = (int)tile - 1;
        uint32_t spins = 0;
        const bool stalled = tile == wait.stallTile;
        while (p >= 0) {
          const uint32_t v = stalled ? 0u : ldRelaxed(&status[(size_t)p * BINS + d]);
          const uint32_t f = v & kFlagMask;
          if (f == 0u) {
            // Plain bounded polling: a predecessor that has claimed its tile
            // is resident and publishes within microseconds.
            if (++spins > wait.spinLimit) {
              atomicOr(errWord, kDevErrLookback);
              break;
            }
            continue;
          }
          excl += v & kValMask;
          if (f == kFlagInc) break;
          --p;
        }
        stRelaxed(&status[(size_t)tile * BINS + d], kFlagInc | ((excl + cnt[k]) & kValMask));
      }
      sDigitStart[d] = exclCnt;
      sGlobal[d] = exclHist + excl - exclCnt;
    }
    exclCnt += cnt[k];
    exclHist += hv[k];
  }
  __syncthreads();

  // Reorder the tile by digit in shared memory.
#pragma unroll
  for (int i = 0; i < IPT; ++i) {
    const uint32_t d = dig[i];
    if (d < (uint32_t)BINS) sItems[sDigitStart[d] + sWarp[warp][d] + off[i]] = item[i];
  }
  __syncthreads();
  const uint32_t valid = min((uint32_t)TILE, n - tileBase);
  for (uint32_t p = tid; p < valid; p += T) {
    const uint2 it = sItems[p];
    const uint32_t d = (it.x >> shift) & mask;
    // Inside [0, n) whenever the digit histogram counts this input (always,
    // unless a corrupted step left the engine's pairs and histogram apart).
    const uint32_t dst = sGlobal[d] + p;
    if (dst < n) out[dst] = it;
    else if (errWord) atomicOr(errWord, kDevErrOrder);
  }
}

template <int BITS>
__global__ void __launch_bounds__(256)
histogramKernel(const uint2* __restrict__ in, uint32_t n, uint32_t passes, uint32_t digitBits,
                uint32_t m0, uint32_t m1, uint32_t m2, uint32_t m3, uint32_t* __restrict__ hist) {
  constexpr int BINS = 1 << BITS;
  __shared__ uint32_t sh[4 * BINS];
  for (int k = threadIdx.x; k < 4 * BINS; k += blockDim.x) sh[k] = 0u;
  __syncthreads();
  const uint32_t masks[4] = {m0, m1, m2, m3};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t key = in[i].x;
    for (uint32_t p = 0; p < passes; ++p) atomicAdd(&sh[p * BINS + ((key >> (p * digitBits)) & masks[p])], 1u);
  }
  __syncthreads();
  for (uint32_t k = threadIdx.x; k < passes * BINS; k += blockDim.x)
    if (sh[k]) atomicAdd(&hist[k], sh[k]);
}

uint32_t passMask(const SortPlan& p, uint32_t pass) {
  uint32_t lo = p.shift[pass];
  uint32_t width = std::min(p.digitBits, p.bits > lo ? p.bits - lo : 0u);
  return width >= 32 ? 0xffffffffu : ((1u << width) - 1u);
}

}  // namespace

SortPlan makeSortPlan(uint32_t n, uint32_t bits, uint32_t maxDigitBits) {
  SortPlan p;
  p.n = n;
  p.bits = std::max(1u, std::min(bits, 32u));
  maxDigitBits = std::max(4u, std::min(maxDigitBits, 9u));
  // At most 4 passes (the plan's shift table and the hash kernel's
  // histograms): narrow digits on wide keys become wider digits.
  p.passes = std::min(4u, (p.bits + maxDigitBits - 1) / maxDigitBits);
  p.digitBits = std::max(4u, (p.bits + p.passes - 1) / p.passes);
  p.bins = 1u << p.digitBits;
  p.tiles = (n + sortTileFor(p.digitBits) - 1) / sortTileFor(p.digitBits);
  for (uint32_t k = 0; k < p.passes; ++k) p.shift[k] = k * p.digitBits;
  return p;
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

size_t sortScratchBytes(const SortPlan& p, bool withTmp) {
  size_t b = 0;
  b += align256((size_t)p.passes * p.bins * 4);
  b += align256((size_t)p.passes * 4);
  b += align256((size_t)p.passes * std::max(1u, p.tiles) * p.bins * 4);
  if (withTmp) b += align256((size_t)p.n * 8);
  return b;
}

SortScratch carveSortScratch(const SortPlan& p, void* base, bool withTmp) {
  SortScratch s;
  char* c = (char*)base;
  s.hist = (uint32_t*)c; c += align256((size_t)p.passes * p.bins * 4);
  s.counters = (uint32_t*)c; c += align256((size_t)p.passes * 4);
  s.status = (uint32_t*)c; c += align256((size_t)p.passes * std::max(1u, p.tiles) * p.bins * 4);
  s.tmp = nullptr;
  if (withTmp) { s.tmp = (uint2*)c; c += align256((size_t)p.n * 8); }
  s.bytes = (size_t)(c - (char*)base);
  return s;
}

cudaError_t launchOnesweepPass(const SortPlan& p, uint32_t pass, const uint2* in, uint2* out,
                               const SortScratch& s, uint32_t* errWord, cudaStream_t st, const uint32_t* gate) {
  if (p.n == 0) return cudaSuccess;
  const uint32_t shift = p.shift[pass], mask = passMask(p, pass);
  const uint32_t* hist = s.hist + (size_t)pass * p.bins;
  uint32_t* status = s.status + (size_t)pass * p.tiles * p.bins;
  uint32_t* counter = s.counters + pass;
  dim3 grid(p.tiles), block(kSortThreads);
  switch (p.digitBits) {
    case 4: onesweepKernel<4><<<grid, block, 0, st>>>(in, out, p.n, shift, mask, hist, status, counter, errWord, gate, p.wait); break;
    case 5: onesweepKernel<5><<<grid, block, 0, st>>>(in, out, p.n, shift, mask, hist, status, counter, errWord, gate, p.wait); break;
    case 6: onesweepKernel<6><<<grid, block, 0, st>>>(in, out, p.n, shift, mask, hist, status, counter, errWord, gate, p.wait); break;
    case 7: onesweepKernel<7><<<grid, block, 0, st>>>(in, out, p.n, shift, mask, hist, status, counter, errWord, gate, p.wait); break;
    case 8: onesweepKernel<8><<<grid, block, 0, st>>>(in, out, p.n, shift, mask, hist, status, counter, errWord, gate, p.wait); break;
    case 9: onesweepKernel<9><<<grid, block, 0, st>>>(in, out, p.n, shift, mask, hist, status, counter, errWord, gate, p.wait); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launchSortHistogram(const SortPlan& p, const uint2* in, const SortScratch& s, cudaStream_t st) {
  if (p.n == 0) return cudaSuccess;
  uint32_t m[4] = {0, 0, 0, 0};
  for (uint32_t k = 0; k < p.passes; ++k) m[k] = passMask(p, k);
  uint32_t blocks = std::min<uint32_t>((p.n + 255) / 256, 148u * 8u);
  switch (p.digitBits) {
#define BRT_HIST_CASE(B) case B: histogramKernel<B><<<blocks, 256, 0, st>>>(in, p.n, p.passes, p.digitBits, m[0], m[1], m[2], m[3], s.hist); break;
    BRT_HIST_CASE(4) BRT_HIST_CASE(5) BRT_HIST_CASE(6) BRT_HIST_CASE(7) BRT_HIST_CASE(8) BRT_HIST_CASE(9)
#undef BRT_HIST_CASE
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

uint32_t sortPassMask(const SortPlan& p, uint32_t pass) { return passMask(p, pass); }

}  // namespace brt

// ---------------------------------------------------------------------------
// Standalone C-ABI sort (BehaveRT::RadixSort replacement, radixsort.cu:50-80).

extern "C" size_t brt_radix_sort_scratch_bytes(uint32_t n, uint32_t bits) {
  brt::SortPlan p = brt::makeSortPlan(n, bits, 8);
  return brt::sortScratchBytes(p, true) + 4 /* error word */ + 256;
}

extern "C" int brt_radix_sort_pairs(const uint32_t* pairs_in, uint32_t* pairs_out, uint32_t n, uint32_t bits,
                                    void* scratch, size_t scratch_bytes, void* stream) {
  brt::TraceRange trace(__func__);
  if (n == 0) return BRT_OK;
  if (!pairs_in || !pairs_out || !scratch) { brt::setLastError("brt_radix_sort_pairs: null pointer"); return BRT_ERR_ARG; }
  if ((const void*)pairs_in == (const void*)pairs_out) { brt::setLastError("brt_radix_sort_pairs: in and out must differ"); return BRT_ERR_ARG; }
  if (n > (1u << 30)) { brt::setLastError("brt_radix_sort_pairs: n > 2^30"); return BRT_ERR_CAPACITY; }
  brt::SortPlan p = brt::makeSortPlan(n, bits, 8);
  const size_t need = brt_radix_sort_scratch_bytes(n, bits);
  if (scratch_bytes < need) { brt::setLastError("brt_radix_sort_pairs: scratch too small"); return BRT_ERR_CAPACITY; }
  cudaStream_t st = (cudaStream_t)stream;
  brt::SortScratch s = brt::carveSortScratch(p, scratch, true);
  uint32_t* err = (uint32_t*)((char*)scratch + s.bytes);
  BRT_CUDA_TRY(cudaMemsetAsync(scratch, 0, s.bytes - (size_t)n * 8 + 4, st));
  BRT_CUDA_TRY(cudaMemsetAsync(err, 0, 4, st));
  BRT_CUDA_TRY(brt::launchSortHistogram(p, (const uint2*)pairs_in, s, st));
  // Ping-pong so that the last pass writes pairs_out.
  const uint2* src = (const uint2*)pairs_in;
  for (uint32_t k = 0; k < p.passes; ++k) {
    uint2* dst = (((p.passes - 1 - k) & 1u) == 0u) ? (uint2*)pairs_out : s.tmp;
    BRT_CUDA_TRY(brt::launchOnesweepPass(p, k, src, dst, s, err, st));
    src = dst;
  }
  uint32_t herr = 0;
  BRT_CUDA_TRY(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, st));
  BRT_CUDA_TRY(cudaStreamSynchronize(st));
  if (herr) { brt::setLastError("brt_radix_sort_pairs: look-back spin limit reached"); return BRT_ERR_TIMEOUT; }
  return BRT_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the standalone sort.
//
// Some callers cannot call cudaMalloc: a frame loop or game-engine plugin
// that must not stall (cudaFree synchronises the whole device), code that runs
// under another framework's caching allocator which owns all device memory,
// and hosts that fix their GPU memory budget at start-up.  For them the sort
// scratch lives in one file-scope device array of a fixed size, sized for at
// most kNoAllocMaxPairs pairs.  Every GPU that loads this library holds the
// array (about 10 MiB) until the process exits.
namespace {

constexpr uint32_t kNoAllocMaxPairs = 1u << 20;
constexpr size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }
// Worst case for n <= kNoAllocMaxPairs with 8-bit digits: 4 passes, 256 bins,
// ceil(2^20 / tile) tiles of the smallest tile size; plus the ping-pong pairs
// and the error word.
constexpr size_t kNoAllocTiles = (kNoAllocMaxPairs + brt::kSortMinTile - 1) / brt::kSortMinTile;
constexpr size_t kNoAllocScratchBytes = a256(4 * 256 * 4) + a256(4 * 4) + a256(4 * kNoAllocTiles * 256 * 4) +
                                        a256((size_t)kNoAllocMaxPairs * 8) + 256;

static __device__ __align__(256) unsigned char g_noAllocSortScratch[kNoAllocScratchBytes];

// The array's name is a host-side stand-in in host code, not a device
// address.  The real address is looked up on every call, with the caller's
// device current: the lookup allocates nothing and costs little, and a
// cached address would go stale once the device's primary context is reset
// or released and made again (the module then loads the array elsewhere).
int noAllocScratchAddress(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0) {
    brt::setLastError("brt_radix_sort_pairs_noalloc: no usable current device");
    return BRT_ERR_NODEVICE;
  }
  void* p = nullptr;
  e = cudaGetSymbolAddress(&p, g_noAllocSortScratch);
  if (e != cudaSuccess || !p) {
    brt::setLastError(std::string("brt_radix_sort_pairs_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    return BRT_ERR_CUDA;
  }
  *out = p;
  return BRT_OK;
}

}  // namespace

extern "C" size_t brt_radix_sort_noalloc_max_pairs(void) { return kNoAllocMaxPairs; }

extern "C" int brt_radix_sort_pairs_noalloc(const uint32_t* pairs_in, uint32_t* pairs_out, uint32_t n, uint32_t bits,
                                            void* stream) {
  brt::TraceRange trace(__func__);
  if (n == 0) return BRT_OK;
  if (!pairs_in || !pairs_out) { brt::setLastError("brt_radix_sort_pairs_noalloc: null pointer"); return BRT_ERR_ARG; }
  if ((const void*)pairs_in == (const void*)pairs_out) {
    brt::setLastError("brt_radix_sort_pairs_noalloc: in and out must differ");
    return BRT_ERR_ARG;
  }
  if (n > kNoAllocMaxPairs) {
    brt::setLastError("brt_radix_sort_pairs_noalloc: n exceeds the 1,048,576-pair limit of the static scratch; "
                      "use brt_radix_sort_pairs with caller-allocated scratch");
    return BRT_ERR_CAPACITY;
  }
  brt::SortPlan p = brt::makeSortPlan(n, bits, 8);
  if (brt::sortScratchBytes(p, true) + 256 > kNoAllocScratchBytes) {
    brt::setLastError("brt_radix_sort_pairs_noalloc: plan exceeds the static scratch");
    return BRT_ERR_CAPACITY;
  }
  void* base = nullptr;
  int rc = noAllocScratchAddress(&base);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  brt::SortScratch s = brt::carveSortScratch(p, base, true);
  uint32_t* err = (uint32_t*)((char*)base + s.bytes);
  // The array keeps the previous call's contents: clear the histogram, tile
  // counters, look-back status and error word (the ping-pong half is fully
  // overwritten before it is read).
  BRT_CUDA_TRY(cudaMemsetAsync(base, 0, (size_t)((char*)s.tmp - (char*)base), st));
  BRT_CUDA_TRY(cudaMemsetAsync(err, 0, 4, st));
  BRT_CUDA_TRY(brt::launchSortHistogram(p, (const uint2*)pairs_in, s, st));
  const uint2* src = (const uint2*)pairs_in;
  for (uint32_t k = 0; k < p.passes; ++k) {
    uint2* dst = (((p.passes - 1 - k) & 1u) == 0u) ? (uint2*)pairs_out : s.tmp;
    BRT_CUDA_TRY(brt::launchOnesweepPass(p, k, src, dst, s, err, st));
    src = dst;
  }
  uint32_t herr = 0;
  BRT_CUDA_TRY(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, st));
  BRT_CUDA_TRY(cudaStreamSynchronize(st));
  if (herr) { brt::setLastError("brt_radix_sort_pairs_noalloc: look-back spin limit reached"); return BRT_ERR_TIMEOUT; }
  return BRT_OK;
}
