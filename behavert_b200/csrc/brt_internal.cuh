// brt_internal.cuh -- shared declarations of the CUDA library (not installed).
//
// The whole library is compiled with --fmad=false and IEEE division / square
// root, so every float + - * / sqrt below is one correctly rounded operation
// in the order written.  That is the same operation sequence the reference's
// device functions spell out (Core/common_resources.cu, the *_resources.cu
// files of the plugins), so results are reproducible bit for bit by a host
// build of the same sequence.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/behavert_b200.h"

#include <nvtx3/nvToolsExt.h>

namespace brt {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;
// Sort mode of a fused step (the incremental re-sort's decision word): the
// hash and radix passes run only in the full-sort mode.
constexpr uint32_t kResortFullSort = 1u, kResortIncremental = 2u;

// Device error word bits (set by kernels, read by brt_engine_check_device_error).
constexpr uint32_t kDevErrLookback = 1u;   // onesweep look-back spin limit hit
constexpr uint32_t kDevErrCapacity = 2u;   // a per-kernel capacity check fired
constexpr uint32_t kDevErrOrder = 4u;      // pipeline invariant violated

// Per-flock parameters as the kernels read them (one entry per flock).
struct FlockDev {
  // geometry: periodic cube [0, L)^3, G cells per side of size cell
  uint32_t G, C, cellBase, agentBase, n;
  float L, cell;
  // Proximity3D
  float radius;
  float r2thr;          // d2 <= r2thr  <=>  !(sqrtf(d2) > radius)
  uint32_t M, maxPerCell;
  int32_t useKnn;
  // OpenSteerWrapper
  float maxSpeed, maxForce, mass, minR;
  float sep[3], ali[3], coh[3];
  int32_t use2D;
  // BehaviorClustering
  uint32_t F;
  float relax;
  float clus, aclus;
  float simStats[3];
  float avgCtl;
  // obstacles
  uint32_t numObstacles;
  float obsW;
  uint32_t obsBase;     // first entry in the engine-wide obstacle table
  float invCell;        // 1 / cell when cell is a power of two (exact), else 0
  // inBoidNeighborhood as exact squared-distance tests:
  //   dist < minR  <=>  d2 < minT,   dist > maxR_b  <=>  d2 > maxT_b
  float minT, sepT, aliT, cohT;
  // Square of -max(cosMaxAngle) when every cosMaxAngle < -1, else 0: for an
  // agent with |forward|^2 * 1.002 below it, every finite cosine passes the
  // angle test, which then only rejects NaN (a zero offset).
  float cosBound2;
  // SchoolingParams (0: flocking law; 1: animateSchool; 2: split path)
  int32_t school;
  float schTheta, schRr, schRp, schEta, schWa, schWo, schS, schRand;
  uint32_t schSeed;
};

// ---------------------------------------------------------------------------
// float3 helpers in the reference's operation order (cutil_math semantics,
// normalize = v * (1 / sqrtf(dot(v, v)))).
struct f3 { float x, y, z; };
__host__ __device__ __forceinline__ f3 mk3(float x, float y, float z) { f3 r; r.x = x; r.y = y; r.z = z; return r; }
__host__ __device__ __forceinline__ f3 add3(f3 a, f3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ f3 sub3(f3 a, f3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ f3 mul3(f3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ __forceinline__ f3 div3(f3 a, float s) { return mk3(a.x / s, a.y / s, a.z / s); }
__host__ __device__ __forceinline__ float dot3(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ float len3(f3 a) { return sqrtf(dot3(a, a)); }
__host__ __device__ __forceinline__ f3 normalize3(f3 v) { float inv = 1.0f / sqrtf(dot3(v, v)); return mul3(v, inv); }
__host__ __device__ __forceinline__ float clampf(float f, float a, float b) { return fmaxf(a, fminf(f, b)); }
__host__ __device__ __forceinline__ f3 xyz(float4 v) { return mk3(v.x, v.y, v.z); }

// envgrid3d_resources.cu:60-84 with origin 0 and clamping to the grid.
// x / cell for a power-of-two cell is computed as x * (1 / cell): the
// reciprocal is exact, and the product and the quotient are the correctly
// rounded values of the same real number, so they agree bit for bit (NaN,
// infinities and subnormals included) at a fraction of an IEEE division.
__device__ __forceinline__ int gridCoordQuotient(float x, const FlockDev& fl) {
  int g = (int)floorf(x / fl.cell);
  return max(0, min(g, (int)fl.G - 1));
}
__device__ __forceinline__ int gridCoord(float x, const FlockDev& fl) {
  const float u = fl.invCell != 0.0f ? x * fl.invCell : x / fl.cell;
  int g = (int)floorf(u);
  return max(0, min(g, (int)fl.G - 1));
}

// Neighbour cell through offset o from home coordinate g, with its image shift.
__device__ __forceinline__ int wrapCoord(int c, uint32_t G) {
  return c < 0 ? c + (int)G : (c >= (int)G ? c - (int)G : c);
}
// Image shift of the neighbour cell g + o (o in {-1, 0, 1}) seen from home
// coordinate g: -L when it wraps below 0, +L when it wraps past G - 1.
// Written on the unwrapped coordinate: the equivalent form
// (o < 0 && g == 0) ? -L : ((o > 0 && g == G - 1) ? L : 0) was compiled
// wrongly for sm_100a at -O3 (nvcc 12.9) when o came from lane arithmetic
// (it returned +L for g = 0, o = +1); a probe checked this form over every
// (g, o) at the seams and in the interior.
__device__ __forceinline__ float imageShift(int g, int o, uint32_t G, float L) {
  const int c = g + o;
  return c < 0 ? -L : (c >= (int)G ? L : 0.0f);
}

// Image shift of a listed neighbour from the two cell coordinates (the
// neighbour is at most one cell away modulo the wrap, and G >= 3): a cell
// difference above 1 means the neighbour is across the lower seam, below -1
// across the upper one.  Written on the difference for the same reason as
// imageShift (the comparison form miscompiled in the same probe).
__device__ __forceinline__ float imageShiftCells(int gi, int gj, uint32_t G, float L) {
  (void)G;
  const int d = gj - gi;
  return d > 1 ? -L : (d < -1 ? L : 0.0f);
}

// Relaxed GPU-scope load and store: the look-back words of the radix passes
// and of the re-sort's cell scan, polled and published across CTAs.
__device__ __forceinline__ uint32_t ldRelaxed(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void stRelaxed(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Flock of a sorted slot (flocks own contiguous slot ranges).
// A cell's sorted-slot range [start, end) as the neighbour scans use it:
// empty unless it lies inside the flock's slots.  A well-formed step always
// passes; after a corrupted one (a look-back wait that ran out, reported
// through the device error word) the words can be stale or torn, and a scan
// must never follow them out of the arrays.
__device__ __forceinline__ bool usableRange(const FlockDev& fl, uint32_t start, uint32_t end) {
  return start != kEmpty && end > start && start >= fl.agentBase && end <= fl.agentBase + fl.n;
}

__device__ __forceinline__ uint32_t flockOfSlot(const uint32_t* __restrict__ agentBase, uint32_t nflocks, uint32_t slot) {
  uint32_t lo = 0, hi = nflocks;  // agentBase has nflocks+1 entries
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (__ldg(&agentBase[mid]) <= slot) lo = mid; else hi = mid;
  }
  return lo;
}

// ---------------------------------------------------------------------------
// Sort plan shared by the engine and the standalone entry point.
// Bound of every decoupled look-back wait (onesweep passes, the incremental
// re-sort's cell scan): polls of a predecessor's unpublished status word
// before the tile gives up, records kDevErrLookback and goes on (the host
// then reports BRT_ERR_TIMEOUT).  About a second at the default.
// stallTile names one tile whose look-back polls as if its predecessor never
// published (a status word that nothing sets), so that tests can make a wait
// run out on purpose; kNoStallTile in normal use.
constexpr uint32_t kDefaultSpinLimit = 1u << 21;
constexpr uint32_t kNoStallTile = 0xFFFFFFFFu;
struct LookbackWait {
  uint32_t spinLimit = kDefaultSpinLimit;
  uint32_t stallTile = kNoStallTile;
};

struct SortPlan {
  uint32_t n = 0, bits = 0, passes = 0, digitBits = 0, bins = 0, tiles = 0;
  uint32_t shift[4] = {0, 0, 0, 0};
  LookbackWait wait;
};
constexpr uint32_t kSortThreads = 256;
// Items a thread ranks per tile: 16, or 8 for 9-bit digits, whose per-warp
// digit counters would not fit beside a 4096-item tile in shared memory.
__host__ __device__ constexpr uint32_t sortItemsFor(uint32_t digitBits) { return digitBits >= 9 ? 8u : 16u; }
__host__ __device__ constexpr uint32_t sortTileFor(uint32_t digitBits) { return kSortThreads * sortItemsFor(digitBits); }
constexpr uint32_t kSortMinTile = kSortThreads * 8u;

SortPlan makeSortPlan(uint32_t n, uint32_t bits, uint32_t maxDigitBits);
// Scratch layout inside one allocation.
struct SortScratch {
  uint32_t* hist;      // passes * bins
  uint32_t* counters;  // passes (tile counters)
  uint32_t* status;    // passes * tiles * bins
  uint2* tmp;          // n pairs (ping-pong), may be null for the engine
  size_t bytes;
};
size_t sortScratchBytes(const SortPlan& p, bool withTmp);
SortScratch carveSortScratch(const SortPlan& p, void* base, bool withTmp);

// Launch one onesweep pass.
// gate (optional): the pass runs only if *gate == kResortFullSort.
cudaError_t launchOnesweepPass(const SortPlan& p, uint32_t pass, const uint2* in, uint2* out,
                               const SortScratch& s, uint32_t* errWord, cudaStream_t st,
                               const uint32_t* gate = nullptr);
// Histogram of all passes' digits (standalone sort only; the engine fuses it
// into the hash kernel).
cudaError_t launchSortHistogram(const SortPlan& p, const uint2* in, const SortScratch& s, cudaStream_t st);

// Thread-local error message.
void setLastError(const std::string& msg);
// A named range on a profiler's timeline (NVTX) for the duration of an entry
// point, as the reference timed its kernel calls (Core/DeviceInterface.cu:
// 389-456): the host-side span of the call, nested ranges included.  With no
// tool attached the push and pop cost a few nanoseconds.
struct TraceRange {
  explicit TraceRange(const char* name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};

// A bad argument to entry point `fn`: records "fn: bad arguments" for
// brt_last_error and returns BRT_ERR_ARG.
inline int argError(const char* fn) {
  setLastError(std::string(fn) + ": bad arguments");
  return BRT_ERR_ARG;
}

}  // namespace brt

#define BRT_CUDA_TRY(expr)                                                              \
  do {                                                                                  \
    cudaError_t _e = (expr);                                                            \
    if (_e != cudaSuccess) {                                                            \
      ::brt::setLastError(std::string(#expr) + ": " + cudaGetErrorString(_e));          \
      return BRT_ERR_CUDA;                                                              \
    }                                                                                   \
  } while (0)
