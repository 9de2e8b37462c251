// brt_resort.cu -- the step's sort on (cell, agent id) derived from the
// previous step's sorted order when few agents change cell.
//
// The result is the same permutation the stable radix sort of
// (key, slot) pairs in agent-id order produces (RadixSort, radixsort.cu:50-80:
// keys ascending, ties by agent id).  It relies on the state the previous
// fused step left behind:
//   * canonical slot j holds the agent that was at sorted position j, so the
//     slots are ordered by (previous key, id) and the previous sorted pairs
//     give each slot's previous key;
//   * cellStart/cellEnd still hold the previous step's cell ranges.
// An agent whose cell did not change (a stayer) keeps its order relative to
// the other stayers of its cell; an agent that moved (a mover) is ranked
// inside its new cell against that cell's stayers (binary search on id in
// the cell's previous range, which is id-sorted) and against the cell's
// other movers (a short per-cell list).  Its sorted position is
//   start(cell) + (stayers of the cell with smaller id) + (movers with smaller id),
// start(cell) being the exclusive scan over cells of stayers + movers.
//
// Kernels, in stream order:
//   resortMarkKernel   new keys, stay flags and per-block stayer prefixes,
//                      per-cell mover lists and counts; its last block decides
//                      the mode of this step (incremental, or the full sort
//                      when the previous order is unknown, a cell received more
//                      than kMaxMoversPerCell movers, or more than maxMovers
//                      agents moved) and scans the block stayer counts;
//   [hash + radix passes, which run only in the full-sort mode]
//   resortCellScanKernel  per-cell totals and their exclusive scan
//                      (single pass, warp-wide decoupled look-back, bounded
//                      waits), and each cell's base for its stayers;
//   resortPlaceKernel  every slot's sorted position.
// The reorder kernel then clears the ranges of cells that became empty and
// resets the mover lists of the cells it sees.
#include "brt_kernels.cuh"

namespace brt {
namespace {

constexpr uint32_t kStayBit = 0x80000000u;
// Cell-scan tiles: THREADS threads of ITEMS consecutive cells, chosen per grid
// (cellScanShape) for about kCellScanTilesTarget tiles: enough to fill the
// GPU, few enough that the look-back stays short when every tile reaches it
// at once.  Small grids take 256-thread tiles of 1 to 4 cells a thread, large
// ones 1024-thread tiles of 8 (measured faster than 256 threads of 32).
// On the 1M-agent flock (262,144 cells) a target of 2 * 148 tiles measured
// the same step time and 1 * 148 (8192-cell tiles) 0.7% slower.
constexpr uint32_t kCellScanTilesTarget = 4 * 148;
constexpr uint32_t kLookAgg = 1u << 30;
constexpr uint32_t kLookInc = 2u << 30;
constexpr uint32_t kLookMask = 3u << 30;
constexpr uint32_t kLookVal = (1u << 30) - 1u;

// Stayers among slots [0, x) and [0, x].
__device__ __forceinline__ uint32_t stayersBefore(const ResortArgs& A, uint32_t x) {
  return __ldg(&A.blockStay[x / kResortChunk]) + (__ldg(&A.prefix[x]) & ~kStayBit);
}
__device__ __forceinline__ uint32_t stayersThrough(const ResortArgs& A, uint32_t x) {
  const uint32_t v = __ldg(&A.prefix[x]);
  return __ldg(&A.blockStay[x / kResortChunk]) + (v & ~kStayBit) + (v >> 31);
}

// Exclusive scan of one value per thread across the CTA (THREADS a multiple
// of 32, at most 1024); the CTA total goes to *total.
template <uint32_t THREADS>
__device__ __forceinline__ uint32_t ctaExclusiveScan(uint32_t v, uint32_t* sWarp, uint32_t* total) {
  constexpr uint32_t WARPS = THREADS / 32;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  if (lane == 31) sWarp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const uint32_t w = lane < WARPS ? sWarp[lane] : 0u;
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= (uint32_t)o) wi += y;
    }
    if (lane < WARPS) sWarp[lane] = wi - w;
    if (lane == WARPS - 1) sWarp[WARPS] = wi;
  }
  __syncthreads();
  const uint32_t r = sWarp[warp] + x - v;
  *total = sWarp[WARPS];
  __syncthreads();
  return r;
}

// One block per chunk of kResortChunk slots, kMarkItems slots a thread
// (slot = chunk * kResortChunk + k * kMarkThreads + thread, so loads stay
// coalesced); the within-chunk stayer prefix comes from one warp-wide scan
// of the (sub-chunk, warp) counts.
constexpr uint32_t kMarkThreads = 256;
constexpr uint32_t kMarkItems = kResortChunk / kMarkThreads;
static_assert(kMarkItems * (kMarkThreads / 32) == 32, "one warp scans the (sub-chunk, warp) counts");

// Eight resident blocks an SM (32 registers, a few spilled bytes): the
// 1,024 chunks of the 1M-agent flock then run as one wave on 148 SMs instead
// of 1.15 waves at the unbounded 40 registers (6 blocks an SM).  Measured
// 0.5% off that step; 128 threads of 8 items (one wave without spills)
// measured slower on the batched flocks.
__global__ void __launch_bounds__(kMarkThreads, 8) resortMarkKernel(ResortArgs A, uint32_t blocks, uint32_t cellTiles) {
  __shared__ uint32_t sCount[32];
  __shared__ uint32_t sWarp[kMarkThreads / 32 + 1];
  __shared__ uint32_t sMovers, sMode, sOverflow;
  __shared__ bool sLast;
  if (A.words[kResortWordValid] == 0u) {
    // previous order unknown: the full sort runs
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      A.words[kResortWordMode] = kResortFullSort;
      A.words[kResortWordMovers] = 0u;
      A.words[kResortWordOverflow] = 0u;
    }
    return;
  }
  constexpr uint32_t kWarps = kMarkThreads / 32;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) { sMovers = 0u; sOverflow = 0u; }
  uint32_t slot[kMarkItems], key[kMarkItems];
  bool stay[kMarkItems], mover[kMarkItems];
  uint32_t bal[kMarkItems];
  uint32_t moving = 0;
  // every load before any store: the arrays are not declared disjoint, so a
  // store between them would keep the next item's loads waiting
  float4 p[kMarkItems];
  uint32_t prevKey[kMarkItems];
#pragma unroll
  for (uint32_t k = 0; k < kMarkItems; ++k) {
    slot[k] = blockIdx.x * kResortChunk + k * kMarkThreads + threadIdx.x;
    p[k] = make_float4(0.f, 0.f, 0.f, 0.f);
    prevKey[k] = 0;
    if (slot[k] < A.n) {
      p[k] = __ldg(&A.pos[slot[k]]);
      prevKey[k] = __ldg(&A.prevPairs[slot[k]].x);
    }
  }
#pragma unroll
  for (uint32_t k = 0; k < kMarkItems; ++k) {
    stay[k] = false;
    mover[k] = false;
    key[k] = 0;
    if (slot[k] < A.n) {
      const uint32_t f = A.nflocks == 1 ? 0u : flockOfSlot(A.agentBase, A.nflocks, slot[k]);
      const FlockDev& fl = A.flocks[f];
      const int gx = gridCoord(p[k].x, fl), gy = gridCoord(p[k].y, fl),
                gz = gridCoord(p[k].z, fl);
      key[k] = fl.cellBase + ((uint32_t)gz * fl.G + (uint32_t)gy) * fl.G + (uint32_t)gx;
      stay[k] = key[k] == prevKey[k];
      mover[k] = !stay[k];
    }
    bal[k] = __ballot_sync(0xffffffffu, stay[k]);
    moving += (uint32_t)__popc(__ballot_sync(0xffffffffu, mover[k]));
    if (lane == 0) sCount[k * kWarps + warp] = (uint32_t)__popc(bal[k]);
  }
#pragma unroll
  for (uint32_t k = 0; k < kMarkItems; ++k)
    if (slot[k] < A.n) A.newKey[slot[k]] = key[k];
  // movers: both atomics of every item in flight together
  uint32_t prev[kMarkItems], count[kMarkItems];
#pragma unroll
  for (uint32_t k = 0; k < kMarkItems; ++k) {
    prev[k] = kNoMover;
    count[k] = 0;
    if (mover[k] && key[k] < A.numCells) {
      prev[k] = atomicExch(&A.moverHead[key[k]], slot[k]);
      count[k] = atomicAdd(&A.moverCount[key[k]], 1u);
    }
  }
  __syncthreads();
  if (warp == 0) {
    const uint32_t v = sCount[lane];
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    sCount[lane] = x - v;
    if (lane == 31) A.blockStay[blockIdx.x] = x;
  }
  if (lane == 0 && moving) atomicAdd(&sMovers, moving);
  __syncthreads();
  const uint32_t below = (1u << lane) - 1u;
#pragma unroll
  for (uint32_t k = 0; k < kMarkItems; ++k) {
    if (slot[k] < A.n)
      A.prefix[slot[k]] = (sCount[k * kWarps + warp] + (uint32_t)__popc(bal[k] & below)) | (stay[k] ? kStayBit : 0u);
    if (mover[k]) {
      if (key[k] >= A.numCells) {
        sOverflow = 1u;  // the full sort's reorder reports the bad key
      } else {
        A.moverNext[slot[k]] = prev[k];
        if (count[k] >= kMaxMoversPerCell) sOverflow = 1u;
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (sMovers) atomicAdd(&A.words[kResortWordMovers], sMovers);
    if (sOverflow) atomicOr(&A.words[kResortWordOverflow], 1u);
    __threadfence();
    sLast = atomicAdd(&A.words[kResortWordDone], 1u) == blocks - 1u;
  }
  __syncthreads();
  if (!sLast) return;

  // The last block to finish decides the step's mode and scans the block
  // stayer counts (every other block's writes are visible after its fence).
  __threadfence();
  if (threadIdx.x == 0) {
    const bool incremental = __ldcg(&A.words[kResortWordOverflow]) == 0u &&
                             __ldcg(&A.words[kResortWordMovers]) <= A.maxMovers;
    sMode = incremental ? kResortIncremental : kResortFullSort;
    A.words[kResortWordMode] = sMode;
    A.words[kResortWordMovers] = 0u;
    A.words[kResortWordOverflow] = 0u;
    A.words[kResortWordDone] = 0u;
    // the hash kernel advances the random-stream step when it runs
    if (incremental && A.stepCounter) *A.stepCounter += 1u;
  }
  __syncthreads();
  if (sMode != kResortIncremental) return;
  for (uint32_t k = threadIdx.x; k < cellTiles; k += kMarkThreads) A.tileStatus[k] = 0u;
  if (threadIdx.x == 0) *A.tileCounter = 0u;
  // in-place exclusive scan of the per-block stayer counts; total at [blocks]
  const uint32_t per = (blocks + kMarkThreads - 1) / kMarkThreads;
  const uint32_t lo = threadIdx.x * per, hi = min(blocks, lo + per);
  uint32_t sum = 0;
  for (uint32_t k = lo; k < hi; ++k) sum += __ldcg(&A.blockStay[k]);
  uint32_t total;
  uint32_t run = ctaExclusiveScan<kMarkThreads>(sum, sWarp, &total);
  for (uint32_t k = lo; k < hi; ++k) {
    const uint32_t v = __ldcg(&A.blockStay[k]);
    A.blockStay[k] = run;
    run += v;
  }
  if (threadIdx.x == 0) A.blockStay[blocks] = total;
}

// Agents of cell c after this step: its stayers (the stayers inside its
// previous range) plus the movers it received; *before gets the stayers
// ahead of that range.
__device__ __forceinline__ uint32_t cellTotal(const ResortArgs& A, uint32_t c, uint32_t* before) {
  uint32_t t = __ldg(&A.moverCount[c]);
  *before = 0;
  const uint32_t s = __ldg(&A.cellStart[c]);
  if (s != kEmpty) {
    const uint32_t e = __ldg(&A.cellEnd[c]);
    if (e > s && e <= A.n) {
      *before = stayersBefore(A, s);
      t += stayersThrough(A, e - 1) - *before;
    }
  }
  return t;
}

template <uint32_t THREADS, uint32_t ITEMS>
__global__ void __launch_bounds__(THREADS) resortCellScanKernel(ResortArgs A) {
  __shared__ uint32_t sTile, sPrefix;
  __shared__ uint32_t sWarp[THREADS / 32 + 1];
  if (A.words[kResortWordMode] != kResortIncremental) return;
  if (threadIdx.x == 0) sTile = atomicAdd(A.tileCounter, 1u);
  __syncthreads();
  const uint32_t tile = sTile;
  const uint32_t c0 = tile * THREADS * ITEMS + threadIdx.x * ITEMS;
  uint32_t tot[ITEMS], ahead[ITEMS];
  uint32_t sum = 0;
#pragma unroll
  for (uint32_t k = 0; k < ITEMS; ++k) {
    const uint32_t c = c0 + k;
    ahead[k] = 0;
    tot[k] = c < A.numCells ? cellTotal(A, c, &ahead[k]) : 0u;
    sum += tot[k];
  }
  uint32_t tileTotal;
  const uint32_t excl = ctaExclusiveScan<THREADS>(sum, sWarp, &tileTotal);
  if (threadIdx.x < 32) {
    // Warp-wide look-back: lane k reads predecessor p - k, so one round
    // covers 32 tiles (tiles that start together would otherwise walk back
    // one dependent load per predecessor).
    const uint32_t lane = threadIdx.x;
    uint32_t before = 0;
    if (tile == 0) {
      if (lane == 0) stRelaxed(&A.tileStatus[0], kLookInc | (tileTotal & kLookVal));
    } else {
      if (lane == 0) stRelaxed(&A.tileStatus[tile], kLookAgg | (tileTotal & kLookVal));
      int p = (int)tile - 1;
      uint32_t spins = 0;
      const bool stalled = tile == A.wait.stallTile;
      while (p >= 0) {
        const int q = p - (int)lane;
        // before tile 0 there is nothing: read as an inclusive zero
        const uint32_t v = q >= 0 ? (stalled ? 0u : ldRelaxed(&A.tileStatus[q])) : kLookInc;
        const uint32_t f = v & kLookMask;
        const uint32_t inc = __ballot_sync(0xffffffffu, f == kLookInc);
        const uint32_t unpublished = __ballot_sync(0xffffffffu, f == 0u);
        const uint32_t first = inc ? (uint32_t)__ffs(inc) - 1u : 31u;  // nearest inclusive prefix
        const uint32_t need = first == 31u ? 0xffffffffu : ((2u << first) - 1u);
        if (unpublished & need) {
          // a predecessor that claimed its tile is resident and publishes soon
          if (++spins > A.wait.spinLimit) {
            if (lane == 0) atomicOr(A.errWord, kDevErrLookback);
            break;
          }
          continue;
        }
        uint32_t add = lane <= first ? (v & kLookVal) : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) add += __shfl_xor_sync(0xffffffffu, add, o);
        before += add;
        if (inc) break;
        p -= 32;
      }
      if (lane == 0) stRelaxed(&A.tileStatus[tile], kLookInc | ((before + tileTotal) & kLookVal));
    }
    if (lane == 0) sPrefix = before;
  }
  __syncthreads();
  uint32_t run = sPrefix + excl;
#pragma unroll
  for (uint32_t k = 0; k < ITEMS; ++k) {
    const uint32_t c = c0 + k;
    if (c < A.numCells) {
      A.newStart[c] = run;
      A.stayBase[c] = run - ahead[k];  // a stayer's position is this plus the stayers before it
    }
    run += tot[k];
  }
}

__global__ void __launch_bounds__(256) resortPlaceKernel(ResortArgs A) {
  if (A.words[kResortWordMode] != kResortIncremental) return;
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= A.n) return;
  const uint32_t c = A.newKey[j];
  const uint32_t pj = __ldg(&A.prefix[j]);
  const uint32_t head = A.moverHead[c];
  uint32_t pos;
  if (pj & kStayBit) {
    // a stayer: after the stayers of its cell's previous range that precede it
    pos = A.stayBase[c] + __ldg(&A.blockStay[j / kResortChunk]) + (pj & ~kStayBit);
  } else {
    // a mover: after the stayers of its new cell with smaller ids (binary
    // search in that cell's previous range, which is id-sorted)
    const uint32_t myId = __ldg(&A.id[j]);
    const uint32_t s0 = __ldg(&A.cellStart[c]);
    uint32_t rank = 0;
    if (s0 != kEmpty) {
      const uint32_t e0 = __ldg(&A.cellEnd[c]);
      if (e0 > A.n || e0 <= s0) {  // ranges that do not fit the previous order
        atomicOr(A.errWord, kDevErrOrder);
        return;
      }
      uint32_t lo = s0, hi = e0;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(&A.id[mid]) < myId) lo = mid + 1; else hi = mid;
      }
      rank = (lo == e0 ? stayersThrough(A, e0 - 1) : stayersBefore(A, lo)) - stayersBefore(A, s0);
    }
    pos = A.newStart[c] + rank;
  }
  // and after the cell's movers with smaller ids
  if (head != kNoMover) {
    const uint32_t myId = __ldg(&A.id[j]);
    uint32_t m = head;
    for (uint32_t hops = 0; m != kNoMover && hops < kMaxMoversPerCell; ++hops) {
      if (__ldg(&A.id[m]) < myId) ++pos;
      m = A.moverNext[m];
    }
  }
  if (pos < A.n) A.out[pos] = make_uint2(c, j);
  else atomicOr(A.errWord, kDevErrOrder);
}

}  // namespace

uint32_t resortBlocks(uint32_t n) { return (n + kResortChunk - 1) / kResortChunk; }
// Cells per tile: 256 (1 a thread), 512, 1024 (256 threads) or 8192 (1024 threads of 8).
static uint32_t cellScanTile(uint32_t numCells) {
  for (uint32_t items = 1; items <= 4; items *= 2)
    if ((numCells + 256u * items - 1) / (256u * items) <= kCellScanTilesTarget) return 256u * items;
  return 8192u;
}
uint32_t resortCellTiles(uint32_t numCells) {
  const uint32_t tile = cellScanTile(numCells);
  return (numCells + tile - 1) / tile;
}

cudaError_t launchResortMark(const ResortArgs& A, cudaStream_t st) {
  if (A.n == 0) return cudaSuccess;
  resortMarkKernel<<<resortBlocks(A.n), kMarkThreads, 0, st>>>(A, resortBlocks(A.n), resortCellTiles(A.numCells));
  return cudaGetLastError();
}

cudaError_t launchResortPlace(const ResortArgs& A, cudaStream_t st) {
  if (A.n == 0) return cudaSuccess;
  const uint32_t tiles = resortCellTiles(A.numCells);
  switch (cellScanTile(A.numCells)) {
    case 256: resortCellScanKernel<256, 1><<<tiles, 256, 0, st>>>(A); break;
    case 512: resortCellScanKernel<256, 2><<<tiles, 256, 0, st>>>(A); break;
    case 1024: resortCellScanKernel<256, 4><<<tiles, 256, 0, st>>>(A); break;
    default: resortCellScanKernel<1024, 8><<<tiles, 1024, 0, st>>>(A); break;
  }
  resortPlaceKernel<<<(A.n + 255) / 256, 256, 0, st>>>(A);
  return cudaGetLastError();
}

}  // namespace brt
