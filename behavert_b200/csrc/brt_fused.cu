// brt_fused.cu -- the fused flocking kernel for flocks without kNN
// replacement or clustering steering (those use fusedKernel, brt_kernels.cu).
//
// One thread per sorted slot.  Phase 1 scans the 27 neighbour cells in the
// reference's visit order (Proximity3D_kernel.cu:108-115) into a shared-memory
// list; phase 2 walks the list in list order (once, or with walk 2 twice:
// geometry, then features), accumulating separation, alignment, cohesion
// (OpenSteerWrapper_resources.cu:166-290) and the feature-relaxation sums with
// the features held in registers and each neighbour's feature norm
// precomputed by the reorder kernel (carried in the w of its sorted
// position).  (Folding the sums into the scan itself makes every scan
// iteration pay for the warp's accepting lanes, which measured slower.)
//
// inBoidNeighborhood (OpenSteerWrapper_resources.cu:67-92) is evaluated with
// exact squared-distance thresholds (sqrtf is monotone and correctly rounded):
//   dist < minR <=> d2 < minT,  dist > maxR <=> d2 > maxT.
// When every cosMaxAngle is below -1 and |forward| is small enough, the angle
// test can only reject a NaN cosine; that needs d2 == 0 (or d2 so small that
// the normalised offset may lose its unit length), so those rare candidates,
// and every candidate when the angle test matters, take the exact path.
#include "brt_agent.cuh"
#include "brt_kernels.cuh"

#include <algorithm>

namespace brt {

// List entries are plain sorted slots; the walk recomputes each neighbour's
// periodic image from its position (neighborImage).

// SCAN: 0 the per-agent scans (variants 0-3, chosen at run time), 4 the
// warp-cooperative scan, 5 the cooperative scan that keeps going agent-major
// in windows of register-held rounds while a run has many open agents; each
// its own instantiation so that it gets its own register allocation.
//
// Scan 7 (the cooperative scan with bounding-box culling) stages each run's
// surviving candidates in shared memory after the lists: (R + 1) rounds of
// float4 per warp, from a 16-byte aligned word offset.
constexpr uint32_t kCullBufPerWarp = (kCoopCachedRounds + 1) * 32;
__host__ __device__ constexpr uint32_t cullBufOffsetWords(uint32_t ls, uint32_t Mmax) { return (ls * Mmax + 3u) & ~3u; }
// Scan 8 (the cooperative scan with the kNN replacement, for engines with a
// useKnn flock and maxNeighbors <= 32) keeps each list's distances beside it.
__host__ __device__ constexpr size_t flockSmemBytes(uint32_t block, uint32_t Mmax, int scan) {
  return scan == 7   ? (size_t)cullBufOffsetWords(block + 1, Mmax) * 4 + (size_t)(block / 32) * kCullBufPerWarp * 16
         : scan == 8 ? (size_t)2 * (block + 1) * Mmax * 4
                     : (size_t)(block + (scan >= 4 ? 1u : 0u)) * Mmax * 4;
}

// Phase 2 of the flock kernels: steering and feature sums over agent i's
// list (list[k * ls], k < n; sorted slots in the reference's visit order),
// then the clustering feature update and the integration of sorted slot i
// into canonical slot i.  Shared by flockKernel and tileFlockKernel, so
// every scan variant walks and integrates with the same code.
template <int FP, int P2>
__device__ __forceinline__ void flockWalk(const FusedArgs& A, uint32_t i, const float4 p4, const FlockDev& fl,
                                          const uint32_t* list, uint32_t ls, uint32_t n) {
  const f3 p = xyz(p4);
  // Phase 2: steering and feature sums over the list, in list order.
  const float4 w4 = __ldg(&A.fwdS[i]);
  const float4 a4 = __ldg(&A.accS[i]);
  const f3 fwd = xyz(w4);
  const bool cosFree = dot3(fwd, fwd) * 1.002f < fl.cosBound2;
  const bool sepOn = fl.sep[0] != 0.0f, aliOn = fl.ali[0] != 0.0f, cohOn = fl.coh[0] != 0.0f;
  const uint32_t F = fl.F;
  const bool relaxOn = FP > 0 && fl.relax != 0.0f && F > 0;
  const uint32_t fs4 = A.Fs / 4;
  float fi[FP > 0 ? FP : 1];
  float facc[FP > 0 ? FP : 1];
  float n1 = 0.0f, sumS = 0.0f;
  if (FP > 0) {
    const float4* src = reinterpret_cast<const float4*>(A.featS) + (size_t)i * fs4;
#pragma unroll
    for (int q = 0; q < FP / 4; ++q) {
      const float4 v = (uint32_t)q < fs4 ? __ldg(&src[q]) : make_float4(0.f, 0.f, 0.f, 0.f);
      fi[4 * q + 0] = v.x; fi[4 * q + 1] = v.y; fi[4 * q + 2] = v.z; fi[4 * q + 3] = v.w;
    }
#pragma unroll
    for (int k = 0; k < FP; ++k) facc[k] = 0.0f;
    n1 = p4.w;  // the reorder stores each agent's feature norm in its sorted position's w
  }
  f3 sSep = mk3(0.f, 0.f, 0.f), sAli = mk3(0.f, 0.f, 0.f), sCoh = mk3(0.f, 0.f, 0.f);
  uint32_t cSep = 0, cAli = 0, cCoh = 0;
  const AgentCtx a = makeCtx(p4, w4, fl);
  // One listed neighbour: its image position, forward and features are
  // loaded by the caller so that several neighbours' loads can be in flight.
  auto visitGeom = [&](const float4 q4, const float4 wj) {
    const f3 img = neighborImage(a, q4, fl);
    const float qx = img.x, qy = img.y, qz = img.z;
    const float dx = qx - p.x, dy = qy - p.y, dz = qz - p.z;
    const float d2 = dx * dx + dy * dy + dz * dz;
    bool inS, inA, inC;
    if (cosFree && d2 >= 1e-30f) {
      const bool lo = d2 < fl.minT;
      inS = lo || !(d2 > fl.sepT);
      inA = lo || !(d2 > fl.aliT);
      inC = lo || !(d2 > fl.cohT);
    } else {
      const float dist = sqrtf(d2);
      const f3 nrm = mul3(mk3(dx, dy, dz), 1.0f / dist);
      const float cosA = dot3(fwd, nrm);
      inS = inBoid(dist, cosA, fl.minR, fl.sep[1], fl.sep[2]);
      inA = inBoid(dist, cosA, fl.minR, fl.ali[1], fl.ali[2]);
      inC = inBoid(dist, cosA, fl.minR, fl.coh[1], fl.coh[2]);
    }
    if (sepOn && inS) {
      const float nd2 = -d2;
      sSep = add3(sSep, mk3(dx / nd2, dy / nd2, dz / nd2));
      ++cSep;
    }
    if (aliOn && inA) {
      sAli = add3(sAli, xyz(wj));
      ++cAli;
    }
    if (cohOn && inC) {
      sCoh = add3(sCoh, mk3(qx, qy, qz));
      ++cCoh;
    }
  };
  auto visitFeat = [&](const float* fj, float n2) {
    if (relaxOn) {
      // computeSimilarity's dot product, then acc += s * f_j, in the
      // reference's sequential order.  Scalar on purpose: ptxas -O3 for
      // sm_100a contracts a packed FP32 multiply feeding a packed add into a
      // fused multiply-add even under --fmad=false and with explicit .rn,
      // which would change the rounding.
      float dot = 0.0f;
#pragma unroll
      for (int kk = 0; kk < FP; ++kk) dot += fi[kk] * fj[kk];
      const float s = (dot / (n1 * n2) + 1.0f) / 2.0f;
      sumS += s;
#pragma unroll
      for (int kk = 0; kk < FP; ++kk) facc[kk] += s * fj[kk];
    }
  };
  auto visit = [&](const float4 q4, const float4 wj, const float* fj, float n2) {
    visitGeom(q4, wj);
    visitFeat(fj, n2);
  };
  auto loadFeat = [&](uint32_t j, float* fj) {
    if (relaxOn) {
      const float4* src = reinterpret_cast<const float4*>(A.featS) + (size_t)j * fs4;
#pragma unroll
      for (int qq = 0; qq < FP / 4; ++qq) {
        const float4 v = (uint32_t)qq < fs4 ? __ldg(&src[qq]) : make_float4(0.f, 0.f, 0.f, 0.f);
        fj[4 * qq + 0] = v.x; fj[4 * qq + 1] = v.y; fj[4 * qq + 2] = v.z; fj[4 * qq + 3] = v.w;
      }
    }
  };
  const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
  if (P2 == 0) {
    for (uint32_t k = 0; k < n; ++k) {
      const uint32_t j = list[k * ls];
      const float4 q = __ldg(&A.posS[j]);
      float fj[FP > 0 ? FP : 1];
      float n2 = q.w;  // the neighbour's feature norm
      loadFeat(j, fj);
      visit(q, aliOn ? __ldg(&A.fwdS[j]) : zero4, fj, n2);
    }
  } else if (P2 == 2) {
    // Two walks over the list, geometry first, then the feature sums: every
    // accumulator still sees the neighbours in list order, and each walk
    // keeps only its own accumulators live.
    for (uint32_t k = 0; k < n; ++k) {
      const uint32_t j = list[k * ls];
      visitGeom(__ldg(&A.posS[j]), aliOn ? __ldg(&A.fwdS[j]) : zero4);
    }
    if (relaxOn) {
      for (uint32_t k = 0; k < n; ++k) {
        const uint32_t j = list[k * ls];
        float fj[FP > 0 ? FP : 1];
        loadFeat(j, fj);
        visitFeat(fj, __ldg(&A.posS[j]).w);
      }
    }
  } else {
    for (uint32_t k = 0; k < n; k += 2) {
      const bool two = k + 1 < n;
      const uint32_t j0 = list[k * ls];
      const uint32_t j1 = two ? (list[(k + 1) * ls]) : j0;
      const float4 q0 = __ldg(&A.posS[j0]), q1 = __ldg(&A.posS[j1]);
      const float4 w0 = aliOn ? __ldg(&A.fwdS[j0]) : zero4, w1 = aliOn ? __ldg(&A.fwdS[j1]) : zero4;
      float f0[FP > 0 ? FP : 1], f1[FP > 0 ? FP : 1];
      float n20 = q0.w, n21 = q1.w;
      loadFeat(j0, f0);
      loadFeat(j1, f1);
      visit(q0, w0, f0, n20);
      if (two) visit(q1, w1, f1, n21);
    }
  }
  f3 steer = mk3(0.f, 0.f, 0.f);
  if (sepOn) {
    if (cSep > 0) sSep = normalize3(div3(sSep, (float)cSep));
    steer = add3(mul3(sSep, fl.sep[0]), steer);
  }
  if (aliOn) {
    if (cAli > 0) sAli = normalize3(sub3(div3(sAli, (float)cAli), fwd));
    steer = add3(mul3(sAli, fl.ali[0]), steer);
  }
  if (cohOn) {
    if (cCoh > 0) sCoh = normalize3(sub3(div3(sCoh, (float)cCoh), p));
    steer = add3(mul3(sCoh, fl.coh[0]), steer);
  }
  if (fl.numObstacles && fl.obsW != 0.0f) steer = obstacleSteer(a, fl, A.obstacles, A.obsMask, steer);
  if (FP > 0) {
    if (relaxOn && n > 0 && sumS > 0.0f) {
#pragma unroll
      for (int k = 0; k < FP; ++k)
        if ((uint32_t)k < F) {
          const float mean = facc[k] / sumS;
          fi[k] = fi[k] + fl.relax * (mean - fi[k]);
        }
    }
    float4* dst = reinterpret_cast<float4*>(A.featA) + (size_t)i * fs4;
#pragma unroll
    for (int q = 0; q < FP / 4; ++q)
      if ((uint32_t)q < fs4) dst[q] = make_float4(fi[4 * q], fi[4 * q + 1], fi[4 * q + 2], fi[4 * q + 3]);
  }
  const Integrated r = integrate(a, a4, steer, A.dt, fl);
  A.posA[i] = r.pos;
  A.fwdA[i] = r.fwd;
  A.accA[i] = r.acc;
  A.idA[i] = __ldg(&A.idS[i]);
}

template <int FP, int P2, int MINB, int SCAN>
__global__ void __launch_bounds__(kFlockMaxThreads, MINB) flockKernel(FusedArgs A) {
  extern __shared__ __align__(16) uint32_t sList[];
  const uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = i0 < A.n;
  // The warp-cooperative scans need every lane of the warp; inactive lanes
  // take part read-only (mirroring the last agent) and leave after it.
  constexpr bool coop = SCAN != 0;
  if (!coop && !active) return;
  const uint32_t i = active ? i0 : A.n - 1;
  const uint32_t f = A.nflocks == 1 ? 0u : flockOfSlot(A.agentBase, A.nflocks, i);
  const FlockDev& fl = A.flocks[f];
  const float4 p4 = __ldg(&A.posS[i]);
  const f3 p = xyz(p4);
  const uint32_t G = fl.G;
  // The plain quotient here (the same cell as gridCoord's product): measured,
  // the product at this point changes ptxas's register allocation of the
  // feature-carrying instantiations (116 against 104 spilled bytes) and costs
  // 2% on the 1M-agent flock, while the product everywhere else saves 0.6%
  // there and 2.2% on the batched flocks.
  const int gx = gridCoordQuotient(p.x, fl), gy = gridCoordQuotient(p.y, fl), gz = gridCoordQuotient(p.z, fl);
  const uint32_t M = fl.M;
  uint32_t* list = sList + threadIdx.x;
  // The cooperative scan stores 32 rows of one agent's column per vote: an
  // odd stride puts those rows in distinct shared-memory banks.
  const uint32_t ls = blockDim.x + (SCAN >= 4 ? 1u : 0u);

  // Phase 1: the neighbour list in the reference's visit order.
  (void)M;
  uint32_t n;
  if (SCAN >= 4) {
    const uint32_t key = fl.cellBase + ((uint32_t)gz * G + (uint32_t)gy) * G + (uint32_t)gx;
    if constexpr (SCAN == 7) {
      float4* cbuf = reinterpret_cast<float4*>(sList + cullBufOffsetWords(ls, A.Mmax)) + (threadIdx.x >> 5) * kCullBufPerWarp;
      n = scanNeighborsCooperative<kCoopCachedRounds, 0, true>(active, i, p, key, A.flocks, f, A.cellStart, A.cellEnd,
                                                               A.posS, sList, ls, threadIdx.x & ~31u, cbuf);
    } else if constexpr (SCAN == 8) {
      float* dList = reinterpret_cast<float*>(sList + ls * A.Mmax);
      n = scanNeighborsCooperative<kCoopCachedRounds, kCoopWindowAgents, false, true>(
          active, i, p, key, A.flocks, f, A.cellStart, A.cellEnd, A.posS, sList, ls, threadIdx.x & ~31u, nullptr, dList);
    } else {
      n = scanNeighborsCooperative<kCoopCachedRounds, SCAN == 5 ? kCoopWindowAgents : 0>(
          active, i, p, key, A.flocks, f, A.cellStart, A.cellEnd, A.posS, sList, ls, threadIdx.x & ~31u);
    }
    if (!active) return;
  } else {
    const bool cull = A.cullGate && __ldg(A.cullGate) == 0u;
    n = A.scanVariant == 0 ? scanNeighborsPipelined<4, true>(i, p, fl, A.cellStart, A.cellEnd, A.posS, list, ls, cull)
      : A.scanVariant == 1 ? scanNeighborsPipelined<2, true>(i, p, fl, A.cellStart, A.cellEnd, A.posS, list, ls, cull)
      : A.scanVariant == 2 ? scanNeighborsPipelined<4, false>(i, p, fl, A.cellStart, A.cellEnd, A.posS, list, ls, false)
                           : scanNeighborsFlat(i, p, fl, A.cellStart, A.cellEnd, A.posS, list, ls);
  }
  if (A.lists) {
    uint32_t* out = A.lists + (size_t)i * A.listStride;
    out[0] = n;
    for (uint32_t k = 0; k < n; ++k) out[1 + k] = list[k * ls];
  }

  flockWalk<FP, P2>(A, i, p4, fl, list, ls, n);
}

// Exclusive scan of one value per thread across a kTileThreads block.
__device__ __forceinline__ uint32_t ctaExclusiveScanTile(uint32_t v, uint32_t* sWarp, uint32_t* total) {
  constexpr uint32_t WARPS = kTileThreads / 32;
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

// ---------------------------------------------------------------------------
// Scan variant 6: a persistent work queue over (flock, row segment) tiles.
//
// A tile is up to kTileMaxCells consecutive home cells of one x-row of one
// flock; its agents are one contiguous range of sorted slots.  A block takes
// tiles from an atomic counter, stages the positions of the tile's
// 9 x (cells + 2) neighbour cells (the union of its agents' 27-cell
// neighbourhoods, each cell once) in shared memory, then every thread scans
// its own agent's 27 cells in the reference's visit order out of shared
// memory: a candidate is loaded from global memory once per tile instead of
// once per home cell.  The list is the same as every other scan's (same
// candidates, same order, same test).  A tile whose neighbourhood holds more
// than kTileStage candidates (dense blobs) is scanned by the warp-cooperative
// scan from global memory instead.  Phase 2 is flockWalk, as for flockKernel.
constexpr uint32_t kTileTable = 9 * (kTileMaxCells + 2);
constexpr uint32_t kTileStage = 1024;

// Agent `self`'s list from the staged tile: sCnt / sOff per table entry
// e = ((oy + 1) * 3 + (oz + 1)) * W + column, column = gx - x0 + 1 + ox.
__device__ __forceinline__ uint32_t scanTileStaged(uint32_t self, f3 p, int gx, int gy, int gz, uint32_t x0, uint32_t W,
                                                   const FlockDev& fl, const float4* sStage, const uint32_t* sOff,
                                                   const uint32_t* sCnt, uint32_t* list, uint32_t ls) {
  const uint32_t M = fl.M;
  const float thr = fl.r2thr;
  uint32_t n = 0;
  for (int ox = -1; ox <= 1; ++ox) {
    const uint32_t col = (uint32_t)(gx - (int)x0 + 1 + ox);
    const float sx = imageShift(gx, ox, fl.G, fl.L);
    for (int oy = -1; oy <= 1; ++oy) {
      const float sy = imageShift(gy, oy, fl.G, fl.L);
      for (int oz = -1; oz <= 1; ++oz) {
        const float sz = imageShift(gz, oz, fl.G, fl.L);
        const uint32_t e = (uint32_t)((oy + 1) * 3 + (oz + 1)) * W + col;
        const uint32_t cnt = sCnt[e], base = sOff[e];
        for (uint32_t k = 0; k < cnt; ++k) {
          const float4 q = sStage[base + k];
          const uint32_t slot = __float_as_uint(q.w);
          const float dx = (q.x + sx) - p.x, dy = (q.y + sy) - p.y, dz = (q.z + sz) - p.z;
          const float d2 = dx * dx + dy * dy + dz * dz;
          if (!(d2 > thr) && slot != self) {
            list[(n++) * ls] = slot;
            if (n == M) return n;
          }
        }
      }
    }
  }
  return n;
}

template <int FP, int P2>
__global__ void __launch_bounds__(kTileThreads, 4) tileFlockKernel(FusedArgs A) {
  extern __shared__ uint32_t sList[];  // (kTileThreads + 1) * Mmax words, a column per thread
  __shared__ float4 sStage[kTileStage];
  __shared__ uint32_t sOff[kTileTable], sCnt[kTileTable], sBeg[kTileTable];
  __shared__ uint32_t sScan[kTileThreads / 32 + 1];
  __shared__ uint32_t sTile, sLo, sHi, sStaged;
  constexpr uint32_t kPer = (kTileTable + kTileThreads - 1) / kTileThreads;  // table entries a thread counts
  const uint32_t tid = threadIdx.x, lane = tid & 31u;
  const uint32_t ls = kTileThreads + 1;
  for (;;) {
    if (tid == 0) sTile = atomicAdd(A.tileCounter, 1u);
    __syncthreads();
    const uint32_t t = sTile;
    if (t >= A.numTiles) return;
    const uint4 d = __ldg(&A.tiles[t]);
    const uint32_t f = d.x, ty = d.y & 0xFFFFu, tz = d.y >> 16, x0 = d.z & 0xFFFFu, R = d.z >> 16;
    const FlockDev& fl = A.flocks[f];
    const uint32_t G = fl.G;
    const uint32_t W = R + 2;
    // the tile's slot range [lo, hi): its home cells' ranges are consecutive
    if (tid < 32) {
      uint32_t lo = 0xFFFFFFFFu, hi = 0u;
      if (lane < R) {
        const uint32_t h = fl.cellBase + (tz * G + ty) * G + x0 + lane;
        const uint32_t st = __ldg(&A.cellStart[h]), en = __ldg(&A.cellEnd[h]);
        if (usableRange(fl, st, en)) { lo = st; hi = en; }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xFFFFFFFFu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xFFFFFFFFu, hi, o));
      }
      if (lane == 0) { sLo = lo; sHi = hi; }
    }
    // the table: counts in table order, their exclusive prefix, staged flags
    uint32_t cnt[kPer], beg[kPer];
    uint32_t mine = 0;
#pragma unroll
    for (uint32_t r = 0; r < kPer; ++r) {
      const uint32_t e = tid * kPer + r;
      cnt[r] = 0;
      beg[r] = 0;
      if (e < 9 * W) {
        const uint32_t row = e / W, col = e - row * W;
        const int oy = (int)(row / 3) - 1, oz = (int)(row % 3) - 1;
        const int cx = wrapCoord((int)x0 - 1 + (int)col, G), cy = wrapCoord((int)ty + oy, G), cz = wrapCoord((int)tz + oz, G);
        const uint32_t h = fl.cellBase + ((uint32_t)cz * G + (uint32_t)cy) * G + (uint32_t)cx;
        const uint32_t st = __ldg(&A.cellStart[h]);
        uint32_t en = __ldg(&A.cellEnd[h]);
        if (usableRange(fl, st, en)) {
          if (fl.maxPerCell && en - st > fl.maxPerCell) en = st + fl.maxPerCell;
          cnt[r] = en - st;
          beg[r] = st;
        }
      }
      mine += cnt[r];
    }
    uint32_t total;
    uint32_t off = ctaExclusiveScanTile(mine, sScan, &total);
#pragma unroll
    for (uint32_t r = 0; r < kPer; ++r) {
      const uint32_t e = tid * kPer + r;
      if (e < kTileTable) {
        sOff[e] = off;
        sCnt[e] = cnt[r];
        sBeg[e] = beg[r];
      }
      off += cnt[r];
    }
    if (tid == 0) sStaged = total <= kTileStage ? total : 0xFFFFFFFFu;
    __syncthreads();
    const uint32_t lo = sLo, hi = sHi;
    const bool staged = sStaged != 0xFFFFFFFFu;
    if (lo < hi && staged) {
      // copy the candidates: entry of q by binary search on the offsets
      const uint32_t entries = 9 * W;
      for (uint32_t q = tid; q < total; q += kTileThreads) {
        uint32_t a = 0, b = entries;  // last entry with sOff <= q
        while (b - a > 1) {
          const uint32_t m = (a + b) >> 1;
          if (sOff[m] <= q) a = m; else b = m;
        }
        const uint32_t slot = sBeg[a] + (q - sOff[a]);
        const float4 v = __ldg(&A.posS[slot]);
        sStage[q] = make_float4(v.x, v.y, v.z, __uint_as_float(slot));
      }
    }
    __syncthreads();
    for (uint32_t base = lo; base < hi; base += kTileThreads) {
      const uint32_t i0 = base + tid;
      const bool active = i0 < hi;
      const uint32_t i = active ? i0 : hi - 1;  // inactive lanes mirror the last agent (read-only)
      const float4 p4 = __ldg(&A.posS[i]);
      const f3 p = xyz(p4);
      const int gx = gridCoord(p.x, fl), gy = gridCoord(p.y, fl), gz = gridCoord(p.z, fl);
      uint32_t n = 0;
      if (staged) {
        // an agent outside the tile's cells only follows a corrupted step
        // (reported by the device error word): no list, no read past the table
        const bool inTile = gx >= (int)x0 && gx < (int)(x0 + R) && gy == (int)ty && gz == (int)tz;
        if (active && inTile) n = scanTileStaged(i, p, gx, gy, gz, x0, W, fl, sStage, sOff, sCnt, sList + tid, ls);
      } else {
        const uint32_t key = fl.cellBase + ((uint32_t)gz * G + (uint32_t)gy) * G + (uint32_t)gx;
        n = scanNeighborsCooperative<kCoopCachedRounds, kCoopWindowAgents>(active, i, p, key, A.flocks, f, A.cellStart,
                                                                            A.cellEnd, A.posS, sList, ls, tid & ~31u);
      }
      if (active) {
        uint32_t* list = sList + tid;
        if (A.lists) {
          uint32_t* out = A.lists + (size_t)i * A.listStride;
          out[0] = n;
          for (uint32_t k = 0; k < n; ++k) out[1 + k] = list[k * ls];
        }
        flockWalk<FP, P2>(A, i, p4, fl, list, ls, n);
      }
      __syncwarp();
    }
    __syncthreads();  // the next tile reuses the staging and the table
  }
}

namespace {
template <int FP, int SCAN>
void launchFlockScan(const FusedArgs& A, uint32_t blocks, uint32_t block, size_t smem, int phase2, int regs,
                     cudaStream_t st) {
  if constexpr (SCAN == 0) {
    if (phase2 == 1) {
      if (regs > 64) flockKernel<FP, 1, 2, 0><<<blocks, block, smem, st>>>(A);
      else flockKernel<FP, 1, 4, 0><<<blocks, block, smem, st>>>(A);
      return;
    }
  }
  if constexpr (SCAN >= 4 && FP > 0) {
    if (phase2 == 2) {
      if (regs <= 48) flockKernel<FP, 2, 5, SCAN><<<blocks, block, smem, st>>>(A);
      else flockKernel<FP, 2, 4, SCAN><<<blocks, block, smem, st>>>(A);
      return;
    }
  }
  if constexpr (SCAN >= 4) {
    if (regs <= 40) { flockKernel<FP, 0, 6, SCAN><<<blocks, block, smem, st>>>(A); return; }
    if (regs <= 48) { flockKernel<FP, 0, 5, SCAN><<<blocks, block, smem, st>>>(A); return; }
  }
  if (regs > 64) flockKernel<FP, 0, 2, SCAN><<<blocks, block, smem, st>>>(A);
  else flockKernel<FP, 0, 4, SCAN><<<blocks, block, smem, st>>>(A);
}
template <int FP>
cudaError_t launchFlockFP(const FusedArgs& A, uint32_t blocks, uint32_t block, size_t smem, int phase2, int regs,
                          cudaStream_t st) {
  if (A.scanVariant == 4) launchFlockScan<FP, 4>(A, blocks, block, smem, phase2, regs, st);
  else if (A.scanVariant == 5) launchFlockScan<FP, 5>(A, blocks, block, smem, phase2, regs, st);
  else if (A.scanVariant == 7) launchFlockScan<FP, 7>(A, blocks, block, smem, phase2, regs, st);
  else if (A.scanVariant == 8) launchFlockScan<FP, 8>(A, blocks, block, smem, phase2, regs, st);
  else launchFlockScan<FP, 0>(A, blocks, block, smem, phase2, regs, st);
  return cudaGetLastError();
}
template <int FP, int SCAN>
cudaError_t configureCoopScan(int smem) {
  const void* fns[4] = {(const void*)flockKernel<FP, 0, 4, SCAN>, (const void*)flockKernel<FP, 0, 2, SCAN>,
                        (const void*)flockKernel<FP, 0, 5, SCAN>, (const void*)flockKernel<FP, 0, 6, SCAN>};
  for (const void* fn : fns) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
  }
  if constexpr (FP > 0) {
    const void* split[2] = {(const void*)flockKernel<FP, 2, 4, SCAN>, (const void*)flockKernel<FP, 2, 5, SCAN>};
    for (const void* fn : split) {
      cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}
template <int FP>
cudaError_t configureFlockFP(int smem, int smemCull, int smemKnn) {
  const void* fns[4] = {(const void*)flockKernel<FP, 0, 4, 0>, (const void*)flockKernel<FP, 1, 4, 0>,
                        (const void*)flockKernel<FP, 0, 2, 0>, (const void*)flockKernel<FP, 1, 2, 0>};
  for (const void* fn : fns) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
  }
  cudaError_t e = configureCoopScan<FP, 4>(smem);
  if (e == cudaSuccess) e = configureCoopScan<FP, 5>(smem);
  if (e == cudaSuccess) e = configureCoopScan<FP, 8>(smemKnn);
  return e == cudaSuccess ? configureCoopScan<FP, 7>(smemCull) : e;
}
}  // namespace

// phase2 1 walks the list two neighbours at a time with their loads issued
// together (per-agent scans only); phase2 2 walks it twice, geometry then
// feature sums (cooperative scan with features only); otherwise one walk,
// one neighbour at a time.  block: threads per block, a multiple of 32
// in [32, 256].  regs: the register budget a thread is compiled for, 128 (2
// resident 256-thread blocks per SM), 64 (4 blocks), or for the cooperative
// scan also 48 and 40 (5 and 6 blocks, more resident warps for some spills).
namespace {
template <int FP>
cudaError_t launchTileFP(const FusedArgs& A, int phase2, cudaStream_t st) {
  const size_t smem = (size_t)(kTileThreads + 1) * A.Mmax * 4;
  cudaError_t e = cudaMemsetAsync(A.tileCounter, 0, 4, st);
  if (e != cudaSuccess) return e;
  if (FP > 0 && phase2 == 2) tileFlockKernel<FP, 2><<<A.tileBlocks, kTileThreads, smem, st>>>(A);
  else tileFlockKernel<FP, 0><<<A.tileBlocks, kTileThreads, smem, st>>>(A);
  return cudaGetLastError();
}
template <int FP>
cudaError_t configureTileFP(int smem) {
  cudaError_t e = cudaFuncSetAttribute(tileFlockKernel<FP, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess && FP > 0)
    e = cudaFuncSetAttribute(tileFlockKernel<FP, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  return e;
}
}  // namespace

// Persistent blocks of the tile kernel a launch should start: the resident
// blocks per SM (shared memory bounds them) times the SMs.
uint32_t tileFlockBlocks(uint32_t Mmax, uint32_t Fs, int smCount) {
  const size_t smem = (size_t)(kTileThreads + 1) * Mmax * 4;
  int per = 0;
  cudaError_t e;
  if (Fs == 0) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, tileFlockKernel<0, 0>, kTileThreads, smem);
  else if (Fs <= 4) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, tileFlockKernel<4, 2>, kTileThreads, smem);
  else if (Fs <= 8) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, tileFlockKernel<8, 2>, kTileThreads, smem);
  else if (Fs <= 16) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, tileFlockKernel<16, 2>, kTileThreads, smem);
  else e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, tileFlockKernel<32, 2>, kTileThreads, smem);
  if (e != cudaSuccess || per < 1) per = 1;
  return (uint32_t)(per * std::max(1, smCount));
}

cudaError_t launchFlock(const FusedArgs& A, int phase2, uint32_t block, int regs, cudaStream_t st) {
  if (A.n == 0) return cudaSuccess;
  if (A.scanVariant == 6) {
    if (!A.tiles || !A.tileCounter || A.tileBlocks == 0) return cudaErrorInvalidValue;
    const uint32_t fp = A.Fs;
    if (fp == 0) return launchTileFP<0>(A, phase2, st);
    if (fp <= 4) return launchTileFP<4>(A, phase2, st);
    if (fp <= 8) return launchTileFP<8>(A, phase2, st);
    if (fp <= 16) return launchTileFP<16>(A, phase2, st);
    return launchTileFP<32>(A, phase2, st);
  }
  if (block < 32 || block > kFlockMaxThreads || block % 32) return cudaErrorInvalidValue;
  const uint32_t blocks = (A.n + block - 1) / block;
  const uint32_t fp = A.Fs;
  const size_t smem = flockSmemBytes(block, A.Mmax, A.scanVariant);
  if (fp == 0) return launchFlockFP<0>(A, blocks, block, smem, phase2, regs, st);
  if (fp <= 4) return launchFlockFP<4>(A, blocks, block, smem, phase2, regs, st);
  if (fp <= 8) return launchFlockFP<8>(A, blocks, block, smem, phase2, regs, st);
  if (fp <= 16) return launchFlockFP<16>(A, blocks, block, smem, phase2, regs, st);
  return launchFlockFP<32>(A, blocks, block, smem, phase2, regs, st);
}

cudaError_t configureFlockKernels(uint32_t Mmax) {
  const int smem = (int)flockSmemBytes(kFlockMaxThreads, Mmax, 5);
  const int smemCull = (int)flockSmemBytes(kFlockMaxThreads, Mmax, 7);
  const int smemKnn = (int)flockSmemBytes(kFlockMaxThreads, std::min<uint32_t>(Mmax, 32), 8);
  cudaError_t e = cudaSuccess;
  if ((e = configureFlockFP<0>(smem, smemCull, smemKnn))) return e;
  if ((e = configureFlockFP<4>(smem, smemCull, smemKnn))) return e;
  if ((e = configureFlockFP<8>(smem, smemCull, smemKnn))) return e;
  if ((e = configureFlockFP<16>(smem, smemCull, smemKnn))) return e;
  if ((e = configureFlockFP<32>(smem, smemCull, smemKnn))) return e;
  const int tsmem = (int)((size_t)(kTileThreads + 1) * Mmax * 4);
  if ((e = configureTileFP<0>(tsmem))) return e;
  if ((e = configureTileFP<4>(tsmem))) return e;
  if ((e = configureTileFP<8>(tsmem))) return e;
  if ((e = configureTileFP<16>(tsmem))) return e;
  return configureTileFP<32>(tsmem);
}

}  // namespace brt
