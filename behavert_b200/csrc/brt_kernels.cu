// brt_kernels.cu -- the per-step pipeline kernels.
//
// Data layout in HBM (N agents over all flocks, C cells over all flocks):
//   canonical state  posA/fwdA/accA float4[N], featA float[N*Fs], idA u32[N]
//                    in the sorted order of the previous step (slot i holds
//                    agent idA[i]); each flock owns a fixed slot range;
//   sorted state     posS/fwdS/accS/featS/idS, the reordered copy the
//                    neighbour pass reads;
//   pairs[2]         (cell key, previous slot) uint2[N], sort ping-pong;
//   cellStart/End    u32[C], 0xFFFFFFFF when empty;
//   similarityStats  float4[N] in agent-id order (only the agent itself
//                    reads it, so it never moves).
// One step: hashKernel -> onesweep passes -> reorderKernel -> fusedKernel.
#include "brt_agent.cuh"
#include "brt_kernels.cuh"

#include <algorithm>

namespace brt {

// ---------------------------------------------------------------------------
// genCalcHashD (envgrid3d_kernel.cu:55-68): key = cellBase + cell hash of the
// agent's position, written at the agent's id so the sort input is in
// agent-id order (the reference hashes the id-ordered position array, and its
// stable sort breaks ties by id).  The value is the agent's current slot.
// The kernel also builds the digit histograms of every sort pass, clears the
// cell ranges and resets the sort's look-back state.
__global__ void __launch_bounds__(256) hashKernel(HashArgs A) {
  extern __shared__ uint32_t sHist[];
  if (A.gate && *A.gate != kResortFullSort) return;  // the incremental re-sort ordered this step
  const uint32_t histWords = A.passes * A.bins;
  for (uint32_t k = threadIdx.x; k < histWords; k += blockDim.x) sHist[k] = 0u;
  __syncthreads();
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t gstride = gridDim.x * blockDim.x;
  for (uint32_t j = gtid; j < A.n; j += gstride) {
    const uint32_t f = A.nflocks == 1 ? 0u : flockOfSlot(A.agentBase, A.nflocks, j);
    const FlockDev& fl = A.flocks[f];
    const float4 p = __ldg(&A.pos[j]);
    const int gx = gridCoord(p.x, fl), gy = gridCoord(p.y, fl), gz = gridCoord(p.z, fl);
    const uint32_t key = fl.cellBase + ((uint32_t)gz * fl.G + (uint32_t)gy) * fl.G + (uint32_t)gx;
    const uint32_t id = __ldg(&A.id[j]);
    A.pairs[id] = make_uint2(key, j);
    for (uint32_t ps = 0; ps < A.passes; ++ps)
      atomicAdd(&sHist[ps * A.bins + ((key >> A.shift[ps]) & A.mask[ps])], 1u);
  }
  uint4* cs = reinterpret_cast<uint4*>(A.cellStart);
  uint4* ce = reinterpret_cast<uint4*>(A.cellEnd);
  const uint4 e4 = make_uint4(kEmpty, kEmpty, kEmpty, kEmpty);
  for (uint32_t c = gtid; c < A.cellWords4; c += gstride) { cs[c] = e4; ce[c] = e4; }
  for (uint32_t k = gtid; k < A.statusWords; k += gstride) A.status[k] = 0u;
  if (gtid < A.passes) A.counters[gtid] = 0u;
  if (gtid == 0 && A.stepCounter) *A.stepCounter += 1u;
  if (gtid == 0 && A.resortValid) *A.resortValid = 0u;
  __syncthreads();
  for (uint32_t k = threadIdx.x; k < histWords; k += blockDim.x)
    if (sHist[k]) atomicAdd(&A.hist[k], sHist[k]);
}

// reorderDataFloat4 (envgrid3d_kernel.cu:110-122) for every registered
// feature in one pass with 128-bit accesses, fused with genericFindCellStartD
// (Proximity3D_kernel.cu:54-84) extended to cellEnd.  Also clears the digit
// histograms for the next step.
__global__ void __launch_bounds__(256) reorderKernel(ReorderArgs A) {
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t gstride = gridDim.x * blockDim.x;
  for (uint32_t k = gtid; k < A.histWords; k += gstride) A.hist[k] = 0u;
  if (A.resortMode && *A.resortMode == kResortIncremental) {
    // the hash kernel did not clear the ranges: clear those of cells that
    // are empty now (the others are written below)
    for (uint32_t c = gtid; c < A.numCells; c += gstride) {
      const uint32_t next = c + 1 < A.numCells ? A.newStart[c + 1] : A.n;
      if (A.newStart[c] == next) { A.cellStart[c] = kEmpty; A.cellEnd[c] = kEmpty; }
    }
  }
  if (gtid == 0 && A.resortValid) *A.resortValid = 1u;
  bool outside = false;  // cell-cull gate: a position of this thread's slots lies outside its cell
  for (uint32_t i = gtid; i < A.n; i += gstride) {
    const uint2 kv = A.pairs[i];
    const uint32_t key = kv.x, ps = kv.y;
    if (ps >= A.n || key >= A.numCells) { atomicOr(A.errWord, kDevErrOrder); continue; }
    const uint32_t prev = i > 0 ? A.pairs[i - 1].x : kEmpty;
    const uint32_t next = i + 1 < A.n ? A.pairs[i + 1].x : kEmpty;
    float4 pos = __ldg(&A.posA[ps]);
    A.fwdS[i] = __ldg(&A.fwdA[ps]);
    A.accS[i] = __ldg(&A.accA[ps]);
    A.idS[i] = __ldg(&A.idA[ps]);
    if (A.prevOut) A.prevOut[i] = ps;
    if (A.fs4) {
      // The feature norm sqrtf(sum f^2) (computeSimilarity's norma,
      // BehaviorClustering_resources.cu:164-175) is the same for every pair
      // an agent takes part in: compute it once here, in the same order.
      // It also goes into the sorted position's w (no kernel reads the w
      // of a position; integration always writes 1), so the list walk gets
      // a neighbour's norm with the neighbour's position.
      const float4* src = reinterpret_cast<const float4*>(A.featA) + (size_t)ps * A.fs4;
      float4* dst = reinterpret_cast<float4*>(A.featS) + (size_t)i * A.fs4;
      float nn = 0.0f;
      for (uint32_t q = 0; q < A.fs4; ++q) {
        const float4 v = __ldg(&src[q]);
        dst[q] = v;
        nn += v.x * v.x;
        nn += v.y * v.y;
        nn += v.z * v.z;
        nn += v.w * v.w;
      }
      pos.w = sqrtf(nn);
    }
    if (A.cullWords && !outside) {
      const FlockDev& fl = A.flocks[A.nflocks == 1 ? 0u : flockOfSlot(A.agentBase, A.nflocks, i)];
      outside = !(pos.x >= 0.0f && pos.x <= fl.L && pos.y >= 0.0f && pos.y <= fl.L && pos.z >= 0.0f && pos.z <= fl.L);
    }
    A.posS[i] = pos;
    if (key != prev) {
      A.cellStart[key] = i;
      if (A.moverHead) { A.moverHead[key] = kNoMover; A.moverCount[key] = 0u; }
    }
    if (key != next) A.cellEnd[key] = i + 1;
  }
  if (A.cullWords) {
    // Scan variants 0 and 1 skip a neighbour cell by the distance from the
    // agent to the cell's face.  That bounds a candidate's distance only when
    // both lie in their hashed cells, which every finite position inside the
    // world does (L is a whole number of cells); a NaN position (clamped into
    // cell 0) or one outside the world (clamped into an edge cell) does not.
    // The last block to finish publishes the OR of all blocks' flags and
    // leaves the accumulator and the ticket at zero for the next launch.
    if (__syncthreads_or(outside) && threadIdx.x == 0) atomicOr(&A.cullWords[0], 1u);
    if (threadIdx.x == 0) {
      __threadfence();
      if (atomicAdd(&A.cullWords[1], 1u) == gridDim.x - 1) {
        A.cullWords[2] = atomicExch(&A.cullWords[0], 0u);
        A.cullWords[1] = 0u;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// The per-agent body shared by the fused pass (one thread per sorted slot).
struct AgentOut {
  Integrated r;
};

__device__ __forceinline__ void loadFeatures(const float* __restrict__ featS, uint32_t Fs, uint32_t i, uint32_t F, float* fi) {
  const float* src = featS + (size_t)i * Fs;
  for (uint32_t k = 0; k < F; ++k) fi[k] = __ldg(&src[k]);
}

// Fused neighbour search + flocking steering + clustering + obstacles +
// feature relaxation + integration.  Lists stay in shared memory
// ([k][thread] layout, odd stride) unless recording is on.  First-M lists
// come from the warp-cooperative windowed scan (every lane of a warp takes
// part; inactive lanes mirror the last agent read-only and leave after it),
// kNN lists (maxNeighbors above a warp) from the per-agent scan.
template <bool KNN>
__global__ void __launch_bounds__(kFusedThreads) fusedKernel(FusedArgs A) {
  extern __shared__ uint32_t sList[];
  const uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = i0 < A.n;
  if (KNN && !active) return;
  const uint32_t i = active ? i0 : A.n - 1;
  const uint32_t f = A.nflocks == 1 ? 0u : flockOfSlot(A.agentBase, A.nflocks, i);
  const FlockDev& fl = A.flocks[f];
  const float4 p4 = __ldg(&A.posS[i]);
  uint32_t* list = sList + threadIdx.x;
  const uint32_t ls = blockDim.x + 1;
  uint32_t n;
  if constexpr (KNN) {
    float distL[BRT_MAX_NEIGHBORS];
    n = buildNeighborList<true>(i, xyz(p4), fl, A.cellStart, A.cellEnd, A.posS, list, ls, distL);
  } else {
    const f3 p = xyz(p4);
    const uint32_t G = fl.G;
    const uint32_t key = fl.cellBase + ((uint32_t)gridCoord(p.z, fl) * G + (uint32_t)gridCoord(p.y, fl)) * G +
                         (uint32_t)gridCoord(p.x, fl);
    n = scanNeighborsCooperative<kCoopCachedRounds, kCoopWindowAgents>(active, i, p, key, A.flocks, f, A.cellStart,
                                                                      A.cellEnd, A.posS, sList, ls, threadIdx.x & ~31u);
    if (!active) return;
  }
  const float4 w4 = __ldg(&A.fwdS[i]);
  const float4 a4 = __ldg(&A.accS[i]);
  if (A.lists) {
    uint32_t* out = A.lists + (size_t)i * A.listStride;
    out[0] = n;
    for (uint32_t k = 0; k < n; ++k) out[1 + k] = list[k * ls];
  }
  const AgentCtx a = makeCtx(p4, w4, fl);
  f3 steer = mk3(0.f, 0.f, 0.f);
  steer = flockingSteer(a, fl, list, ls, n, A.posS, A.fwdS, steer, fl.sep[0] != 0.0f, fl.ali[0] != 0.0f, fl.coh[0] != 0.0f);
  float fi[BRT_MAX_FEATUREDIM];
  float norm1 = 0.0f;
  const uint32_t F = fl.F;
  if (F) {
    loadFeatures(A.featS, A.Fs, i, F, fi);
    norm1 = selfNorm(fi, F);
  }
  if (F && (fl.clus != 0.0f || fl.aclus != 0.0f)) {
    const uint32_t id = __ldg(&A.idS[i]);
    float4 st = A.statsById[id];
    float sims[BRT_MAX_NEIGHBORS];
    steer = clusteringSteer(a, fl, list, ls, n, A.posS, A.fwdS, fi, norm1, A.featS, A.Fs, st, sims, steer);
    A.statsById[id] = st;
  }
  if (fl.numObstacles && fl.obsW != 0.0f) steer = obstacleSteer(a, fl, A.obstacles, A.obsMask, steer);
  if (F) {
    float fo[BRT_MAX_FEATUREDIM];
    relaxFeatures(fl, list, ls, n, fi, norm1, A.featS, A.Fs, fo);
    float* dst = A.featA + (size_t)i * A.Fs;
    for (uint32_t k = 0; k < F; ++k) dst[k] = fo[k];
  }
  const Integrated r = integrate(a, a4, steer, A.dt, fl);
  A.posA[i] = r.pos;
  A.fwdA[i] = r.fwd;
  A.accA[i] = r.acc;
  A.idA[i] = __ldg(&A.idS[i]);
}

// ---------------------------------------------------------------------------
// Stage-wise kernels (the reference's separate functionalities).

// computeNeighborhoods: every agent's list into the list array.  First-M
// lists come from the warp-cooperative windowed scan through shared memory
// (inactive lanes take part read-only), kNN lists from the per-agent scan.
template <bool KNN>
__global__ void __launch_bounds__(128) listsKernel(StageArgs A) {
  extern __shared__ uint32_t sList[];
  const uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = i0 < A.n;
  if (KNN && !active) return;
  const uint32_t i = active ? i0 : A.n - 1;
  const uint32_t f = A.nflocks == 1 ? 0u : flockOfSlot(A.agentBase, A.nflocks, i);
  const FlockDev& fl = A.flocks[f];
  uint32_t* out = A.lists + (size_t)i * A.listStride;
  const f3 p = xyz(__ldg(&A.posS[i]));
  if constexpr (KNN) {
    float distL[BRT_MAX_NEIGHBORS];
    out[0] = buildNeighborList<true>(i, p, fl, A.cellStart, A.cellEnd, A.posS, out + 1, 1, distL);
  } else {
    const uint32_t G = fl.G;
    const uint32_t key = fl.cellBase + ((uint32_t)gridCoord(p.z, fl) * G + (uint32_t)gridCoord(p.y, fl)) * G +
                         (uint32_t)gridCoord(p.x, fl);
    const uint32_t ls = blockDim.x + 1;
    const uint32_t n = scanNeighborsCooperative<kCoopCachedRounds, kCoopWindowAgents>(
        active, i, p, key, A.flocks, f, A.cellStart, A.cellEnd, A.posS, sList, ls, threadIdx.x & ~31u);
    if (!active) return;
    const uint32_t* list = sList + threadIdx.x;
    for (uint32_t k = 0; k < n; ++k) out[1 + k] = list[k * ls];
    out[0] = n;
  }
}

// which: 0 separation, 1 alignment, 2 cohesion, 3 clustering, 4 obstacles
__global__ void __launch_bounds__(128) steerStageKernel(StageArgs A, int which) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const uint32_t f = A.nflocks == 1 ? 0u : flockOfSlot(A.agentBase, A.nflocks, i);
  const FlockDev& fl = A.flocks[f];
  const uint32_t* lst = A.lists + (size_t)i * A.listStride;
  const uint32_t n = lst[0];
  const AgentCtx a = makeCtx(__ldg(&A.posS[i]), __ldg(&A.fwdS[i]), fl);
  const float4 s4 = A.steer[i];
  f3 steer = xyz(s4);
  if (which == 0 && fl.sep[0] != 0.0f) steer = flockingSteer(a, fl, lst + 1, 1, n, A.posS, A.fwdS, steer, true, false, false);
  if (which == 1 && fl.ali[0] != 0.0f) steer = flockingSteer(a, fl, lst + 1, 1, n, A.posS, A.fwdS, steer, false, true, false);
  if (which == 2 && fl.coh[0] != 0.0f) steer = flockingSteer(a, fl, lst + 1, 1, n, A.posS, A.fwdS, steer, false, false, true);
  if (which == 3 && fl.F && (fl.clus != 0.0f || fl.aclus != 0.0f)) {
    float fi[BRT_MAX_FEATUREDIM];
    loadFeatures(A.featS, A.Fs, i, fl.F, fi);
    const float norm1 = selfNorm(fi, fl.F);
    const uint32_t id = __ldg(&A.idS[i]);
    float4 st = A.statsById[id];
    float sims[BRT_MAX_NEIGHBORS];
    steer = clusteringSteer(a, fl, lst + 1, 1, n, A.posS, A.fwdS, fi, norm1, A.featS, A.Fs, st, sims, steer);
    A.statsById[id] = st;
  }
  if (which == 4 && fl.numObstacles && fl.obsW != 0.0f) steer = obstacleSteer(a, fl, A.obstacles, A.obsMask, steer);
  if (which == 5) {
    // The new speed goes to this agent's own forward entry, which no other
    // thread reads in this stage; blendIntoSteeringForce adds the force.
    float speed = a.speed;
    const f3 s = avoidNeighbors(a, fl, lst + 1, 1, n, A.posS, &speed);
    A.fwdW[i] = make_float4(a.fwd.x, a.fwd.y, a.fwd.z, speed);
    steer = add3(s, steer);
  }
  if (which == 6) {
    // moveAwayFromTarget_kernel (OpenSteerWrapper_kernel.cu:185-212): flee the
    // base point, (weight * offset) / distance, nothing beyond twice the
    // radius.  The kernel's acceleration write is overwritten by its own copy
    // of the old value, so the smoothed acceleration is left as it is.  As in
    // the reference: the direct offset (no periodic image), and 0/0 for an
    // agent exactly at the base point.
    f3 s = sub3(a.pos, mk3(A.avoidBase[0], A.avoidBase[1], A.avoidBase[2]));
    const float d = len3(s);
    if (d > A.avoidBaseParams[2] * 2.0f) s = mk3(0.f, 0.f, 0.f);
    steer = add3(div3(mul3(s, A.avoidBaseParams[0]), d), steer);
  }
  A.steer[i] = make_float4(steer.x, steer.y, steer.z, 0.0f);
}

__global__ void __launch_bounds__(128) integrateStageKernel(StageArgs A, float dt) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const uint32_t f = A.nflocks == 1 ? 0u : flockOfSlot(A.agentBase, A.nflocks, i);
  const FlockDev& fl = A.flocks[f];
  const uint32_t* lst = A.lists + (size_t)i * A.listStride;
  const uint32_t n = lst[0];
  const float4 p4 = __ldg(&A.posS[i]), w4 = __ldg(&A.fwdS[i]), a4 = __ldg(&A.accS[i]);
  const AgentCtx a = makeCtx(p4, w4, fl);
  if (fl.F) {
    float fi[BRT_MAX_FEATUREDIM], fo[BRT_MAX_FEATUREDIM];
    loadFeatures(A.featS, A.Fs, i, fl.F, fi);
    const float norm1 = selfNorm(fi, fl.F);
    relaxFeatures(fl, lst + 1, 1, n, fi, norm1, A.featS, A.Fs, fo);
    float* dst = A.featA + (size_t)i * A.Fs;
    for (uint32_t k = 0; k < fl.F; ++k) dst[k] = fo[k];
  }
  const Integrated r = integrate(a, a4, xyz(A.steer[i]), dt, fl);
  A.posA[i] = r.pos;
  A.fwdA[i] = r.fwd;
  A.accA[i] = r.acc;
  A.idA[i] = __ldg(&A.idS[i]);
}

// ---------------------------------------------------------------------------
// State I/O between agent-id order and the canonical slot order.

__global__ void scatterToIdKernel(const float4* __restrict__ src, const uint32_t* __restrict__ id, float4* __restrict__ dst, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[__ldg(&id[i])] = __ldg(&src[i]);
}
__global__ void scatterFeatToIdKernel(const float* __restrict__ src, uint32_t Fs, const uint32_t* __restrict__ id, float* __restrict__ dst, uint32_t F, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t d = __ldg(&id[i]);
  for (uint32_t k = 0; k < F; ++k) dst[(size_t)d * F + k] = __ldg(&src[(size_t)i * Fs + k]);
}
__global__ void loadFeatKernel(const float* __restrict__ src, uint32_t F, float* __restrict__ dst, uint32_t Fs, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (uint32_t k = 0; k < Fs; ++k) dst[(size_t)i * Fs + k] = k < F ? __ldg(&src[(size_t)i * F + k]) : 0.0f;
}
// Permute a float4 feature given in agent-id order into canonical slot order
// (positions keep w = 1, like the reference's position feature).
__global__ void gatherFromIdKernel(const float4* __restrict__ src, const uint32_t* __restrict__ id, float4* __restrict__ dst, uint32_t n, int forceW1) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 v = __ldg(&src[__ldg(&id[i])]);
  if (forceW1) v.w = 1.0f;
  dst[i] = v;
}
__global__ void gatherFeatFromIdKernel(const float* __restrict__ src, uint32_t F, const uint32_t* __restrict__ id, float* __restrict__ dst, uint32_t Fs, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t s = __ldg(&id[i]);
  for (uint32_t k = 0; k < Fs; ++k) dst[(size_t)i * Fs + k] = k < F ? __ldg(&src[(size_t)s * F + k]) : 0.0f;
}
__global__ void hashPairsToOutKernel(const uint2* __restrict__ pairs, const uint32_t* __restrict__ idS, uint32_t* keys, uint32_t* ids, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (keys) keys[i] = pairs[i].x;
  if (ids) ids[i] = __ldg(&idS[i]);
}

// ---------------------------------------------------------------------------
// Launchers.

static inline uint32_t blocksFor(uint32_t n, uint32_t t) { return (n + t - 1) / t; }

cudaError_t launchHash(const HashArgs& A, uint32_t smBlocks, cudaStream_t st) {
  const uint32_t blocks = std::max(1u, std::min(blocksFor(A.n, 256), smBlocks));
  hashKernel<<<blocks, 256, A.passes * A.bins * 4, st>>>(A);
  return cudaGetLastError();
}
cudaError_t launchReorder(const ReorderArgs& A, cudaStream_t st) {
  const uint32_t blocks = std::max(1u, blocksFor(std::max(A.n, A.histWords), 256));
  reorderKernel<<<blocks, 256, 0, st>>>(A);
  return cudaGetLastError();
}
cudaError_t configureFusedKernels(uint32_t Mmax) {
  const int smem = (int)((size_t)(kFusedThreads + 1) * Mmax * 4);
  cudaError_t e = cudaFuncSetAttribute(fusedKernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(fusedKernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(listsKernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(129 * Mmax * 4));
}
cudaError_t launchFused(const FusedArgs& A, bool knn, cudaStream_t st) {
  if (A.n == 0) return cudaSuccess;
  const size_t smem = (size_t)(kFusedThreads + 1) * A.Mmax * 4;
  if (knn) fusedKernel<true><<<blocksFor(A.n, kFusedThreads), kFusedThreads, smem, st>>>(A);
  else fusedKernel<false><<<blocksFor(A.n, kFusedThreads), kFusedThreads, smem, st>>>(A);
  return cudaGetLastError();
}
cudaError_t launchLists(const StageArgs& A, bool knn, cudaStream_t st) {
  if (A.n == 0) return cudaSuccess;
  if (knn) listsKernel<true><<<blocksFor(A.n, 128), 128, 0, st>>>(A);
  else listsKernel<false><<<blocksFor(A.n, 128), 128, (size_t)129 * (A.listStride - 1) * 4, st>>>(A);
  return cudaGetLastError();
}
// Registered per-agent arrays of `words` 32-bit words: slot i of dst takes
// slot index[i * stride] of src (gather), or slot i of src goes to slot
// index[i] of dst (scatter); one thread per word.
__global__ void gatherWordsKernel(const uint32_t* __restrict__ src, const uint32_t* __restrict__ index, uint32_t stride,
                                  uint32_t* __restrict__ dst, uint32_t words, uint32_t n) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)n * words) return;
  const size_t i = t / words, k = t - i * words;
  const uint32_t from = __ldg(&index[i * stride]);
  dst[t] = from < n ? src[(size_t)from * words + k] : 0u;  // a corrupted step's stale index reads nothing
}
__global__ void scatterWordsKernel(const uint32_t* __restrict__ src, const uint32_t* __restrict__ index,
                                   uint32_t* __restrict__ dst, uint32_t words, uint32_t n) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)n * words) return;
  const size_t i = t / words, k = t - i * words;
  dst[(size_t)__ldg(&index[i]) * words + k] = src[t];
}
cudaError_t launchGatherWords(const uint32_t* src, const uint32_t* index, uint32_t stride, uint32_t* dst, uint32_t words,
                              uint32_t n, cudaStream_t st) {
  const size_t total = (size_t)n * words;
  if (total == 0) return cudaSuccess;
  gatherWordsKernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(src, index, stride, dst, words, n);
  return cudaGetLastError();
}
cudaError_t launchScatterWords(const uint32_t* src, const uint32_t* index, uint32_t* dst, uint32_t words, uint32_t n,
                               cudaStream_t st) {
  const size_t total = (size_t)n * words;
  if (total == 0) return cudaSuccess;
  scatterWordsKernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(src, index, dst, words, n);
  return cudaGetLastError();
}

cudaError_t launchSteerStage(const StageArgs& A, int which, cudaStream_t st) {
  if (A.n == 0) return cudaSuccess;
  steerStageKernel<<<blocksFor(A.n, 128), 128, 0, st>>>(A, which);
  return cudaGetLastError();
}
cudaError_t launchIntegrateStage(const StageArgs& A, float dt, cudaStream_t st) {
  if (A.n == 0) return cudaSuccess;
  integrateStageKernel<<<blocksFor(A.n, 128), 128, 0, st>>>(A, dt);
  return cudaGetLastError();
}
cudaError_t launchScatterToId(const float4* src, const uint32_t* id, float4* dst, uint32_t n, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  scatterToIdKernel<<<blocksFor(n, 256), 256, 0, st>>>(src, id, dst, n);
  return cudaGetLastError();
}
cudaError_t launchScatterFeatToId(const float* src, uint32_t Fs, const uint32_t* id, float* dst, uint32_t F, uint32_t n, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  scatterFeatToIdKernel<<<blocksFor(n, 256), 256, 0, st>>>(src, Fs, id, dst, F, n);
  return cudaGetLastError();
}
cudaError_t launchLoadFeat(const float* src, uint32_t F, float* dst, uint32_t Fs, uint32_t n, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  loadFeatKernel<<<blocksFor(n, 256), 256, 0, st>>>(src, F, dst, Fs, n);
  return cudaGetLastError();
}
cudaError_t launchGatherFromId(const float4* src, const uint32_t* id, float4* dst, uint32_t n, bool forceW1, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  gatherFromIdKernel<<<blocksFor(n, 256), 256, 0, st>>>(src, id, dst, n, forceW1 ? 1 : 0);
  return cudaGetLastError();
}
cudaError_t launchGatherFeatFromId(const float* src, uint32_t F, const uint32_t* id, float* dst, uint32_t Fs, uint32_t n, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  gatherFeatFromIdKernel<<<blocksFor(n, 256), 256, 0, st>>>(src, F, id, dst, Fs, n);
  return cudaGetLastError();
}
cudaError_t launchHashPairsOut(const uint2* pairs, const uint32_t* idS, uint32_t* keys, uint32_t* ids, uint32_t n, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  hashPairsToOutKernel<<<blocksFor(n, 256), 256, 0, st>>>(pairs, idS, keys, ids, n);
  return cudaGetLastError();
}

}  // namespace brt
