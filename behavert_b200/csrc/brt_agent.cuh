// brt_agent.cuh -- per-agent device functions shared by the fused pass and
// the stage-wise kernels, so both produce bit-identical results.
//
// Each function cites the reference device code whose operation order it
// keeps.  Positions live in the periodic cube [0, L)^3; a neighbour reached
// through a wrapped cell is used at its image position q + s, s in {-L,0,+L}.
#pragma once

#include "brt_internal.cuh"

namespace brt {

// genericCalcNeighgborhoodD + checkForNeighborsInCell + checkForNeighbor
// (Proximity3D_kernel.cu:89-125, Proximity3D_resources.cu:59-172), periodic.
// Visit order x outermost, y, z innermost; within a cell ascending sorted
// slot; self skipped by slot; accept iff !(sqrtf(d2) > radius), evaluated as
// d2 <= r2thr (sqrtf is monotone and correctly rounded, r2thr is the largest
// float whose root does not exceed the radius).  With kNN off the scan stops
// once M entries are held: later candidates cannot change the list.
template <bool KNN>
__device__ __forceinline__ uint32_t buildNeighborList(uint32_t self, f3 p, const FlockDev& fl,
                                                      const uint32_t* __restrict__ cellStart,
                                                      const uint32_t* __restrict__ cellEnd,
                                                      const float4* __restrict__ posS, uint32_t* list,
                                                      uint32_t ls, float* distList) {
  const int gx = gridCoord(p.x, fl), gy = gridCoord(p.y, fl), gz = gridCoord(p.z, fl);
  const uint32_t M = fl.M;
  // kNN replacement is per flock: an engine may mix kNN and first-M flocks
  const bool knn = KNN && fl.useKnn;
  uint32_t n = 0;
  float maxDistValue = 0.0f;
  for (int ox = -1; ox <= 1; ++ox) {
    const int cx = wrapCoord(gx + ox, fl.G);
    const float sx = imageShift(gx, ox, fl.G, fl.L);
    for (int oy = -1; oy <= 1; ++oy) {
      const int cy = wrapCoord(gy + oy, fl.G);
      const float sy = imageShift(gy, oy, fl.G, fl.L);
      for (int oz = -1; oz <= 1; ++oz) {
        const int cz = wrapCoord(gz + oz, fl.G);
        const float sz = imageShift(gz, oz, fl.G, fl.L);
        const uint32_t h = fl.cellBase + ((uint32_t)cz * fl.G + (uint32_t)cy) * fl.G + (uint32_t)cx;
        const uint32_t start = __ldg(&cellStart[h]);
        uint32_t stop = __ldg(&cellEnd[h]);
        if (!usableRange(fl, start, stop)) continue;
        if (fl.maxPerCell && stop - start > fl.maxPerCell) stop = start + fl.maxPerCell;
        for (uint32_t j = start; j < stop; ++j) {
          if (j == self) continue;
          const float4 q = __ldg(&posS[j]);
          const float dx = (q.x + sx) - p.x, dy = (q.y + sy) - p.y, dz = (q.z + sz) - p.z;
          const float d2 = dx * dx + dy * dy + dz * dz;
          if (!knn) {
            if (d2 > fl.r2thr) continue;
            list[(n++) * ls] = j;
            if (n == M) return n;
          } else {
            const float dist = sqrtf(d2);
            if (dist > fl.radius) continue;
            if (n < M) {
              list[n * ls] = j;
              distList[n] = dist;
              maxDistValue = fmaxf(maxDistValue, dist);
              ++n;
            } else if (dist < maxDistValue) {
              maxDistValue = distList[0];
              uint32_t maxIdx = 0;
              for (uint32_t k = 1; k < n; ++k)
                if (maxDistValue < distList[k]) { maxDistValue = distList[k]; maxIdx = k; }
              list[maxIdx * ls] = j;
              distList[maxIdx] = dist;
            }
          }
        }
      }
    }
  }
  return n;
}

// The same list as buildNeighborList<false>, walked as one flat loop over the
// concatenated candidates of the 27 cells (same visit order).  Lanes of a
// warp whose home cells differ then run the candidate loop in lockstep
// instead of diverging on every cell's own trip count.
__device__ __forceinline__ uint32_t scanNeighborsFlat(uint32_t self, f3 p, const FlockDev& fl,
                                                      const uint32_t* __restrict__ cellStart,
                                                      const uint32_t* __restrict__ cellEnd,
                                                      const float4* __restrict__ posS, uint32_t* list,
                                                      uint32_t ls) {
  const int gx = gridCoord(p.x, fl), gy = gridCoord(p.y, fl), gz = gridCoord(p.z, fl);
  const uint32_t M = fl.M;
  const float thr = fl.r2thr;
  uint32_t n = 0;
  int c = -1;
  uint32_t j = 0, stop = 0;
  float sx = 0.0f, sy = 0.0f, sz = 0.0f;
  for (;;) {
    if (j >= stop) {
      bool found = false;
      while (++c < 27) {
        const int ox = c / 9 - 1, oy = (c / 3) % 3 - 1, oz = c % 3 - 1;
        const int cx = wrapCoord(gx + ox, fl.G), cy = wrapCoord(gy + oy, fl.G), cz = wrapCoord(gz + oz, fl.G);
        const uint32_t h = fl.cellBase + ((uint32_t)cz * fl.G + (uint32_t)cy) * fl.G + (uint32_t)cx;
        const uint32_t start = __ldg(&cellStart[h]);
        uint32_t end = __ldg(&cellEnd[h]);
        if (!usableRange(fl, start, end)) continue;
        if (fl.maxPerCell && end - start > fl.maxPerCell) end = start + fl.maxPerCell;
        j = start;
        stop = end;
        sx = imageShift(gx, ox, fl.G, fl.L);
        sy = imageShift(gy, oy, fl.G, fl.L);
        sz = imageShift(gz, oz, fl.G, fl.L);
        found = true;
        break;
      }
      if (!found) break;
    }
    if (j != self) {
      const float4 q = __ldg(&posS[j]);
      const float dx = (q.x + sx) - p.x, dy = (q.y + sy) - p.y, dz = (q.z + sz) - p.z;
      const float d2 = dx * dx + dy * dy + dz * dz;
      if (!(d2 > thr)) {
        list[(n++) * ls] = j;
        if (n == M) break;
      }
    }
    ++j;
  }
  return n;
}

// The same list as buildNeighborList<false> (same visit order, same test),
// written for memory-level parallelism: for each (x, y) row the three z
// cells' ranges are fetched together, and candidate positions are loaded
// UNROLL at a time before they are tested in order.
//
// With CULL and `cull` set, a neighbour cell is skipped when its box is
// provably farther than the search radius: the distance from p to the shared
// face is exact (p - g*cell and (g+1)*cell - p are Sterbenz-exact for g >= 1,
// within an ulp of 4 otherwise) and any candidate of that cell lies beyond
// the face up to the rounding of its own coordinate, so a margin of 0.01 on
// d^2 cannot drop a candidate that would pass the exact test.  Skipping such
// a cell therefore leaves the list unchanged.  That holds only while every
// position lies in its hashed cell: a NaN position is hashed to cell 0 and
// accepted by every agent that reads it (!(NaN > r2thr)), and a position
// outside the world is clamped into an edge cell.  The caller clears `cull`
// when the step's sorted state holds such a position.
template <int UNROLL, bool CULL>
__device__ __forceinline__ uint32_t scanNeighborsPipelined(uint32_t self, f3 p, const FlockDev& fl,
                                                           const uint32_t* __restrict__ cellStart,
                                                           const uint32_t* __restrict__ cellEnd,
                                                           const float4* __restrict__ posS, uint32_t* list,
                                                           uint32_t ls, bool cull) {
  const int gx = gridCoord(p.x, fl), gy = gridCoord(p.y, fl), gz = gridCoord(p.z, fl);
  const uint32_t M = fl.M;
  const float thr = fl.r2thr;
  // squared distances to the lower / upper faces of the home cell
  float lo2[3], hi2[3];
  if (CULL) {
    const float cl = fl.cell;
    const float lx = p.x - (float)gx * cl, ly = p.y - (float)gy * cl, lz = p.z - (float)gz * cl;
    const float ux = (float)(gx + 1) * cl - p.x, uy = (float)(gy + 1) * cl - p.y, uz = (float)(gz + 1) * cl - p.z;
    lo2[0] = lx * lx; lo2[1] = ly * ly; lo2[2] = lz * lz;
    hi2[0] = ux * ux; hi2[1] = uy * uy; hi2[2] = uz * uz;
  }
  // The candidate-coordinate rounding grows with the world size (ulp of L).
  const float cullThr = thr + 0.01f + 1e-6f * fl.cell * fl.L;
  uint32_t n = 0;
  for (int ox = -1; ox <= 1; ++ox) {
    const int cx = wrapCoord(gx + ox, fl.G);
    const float sx = imageShift(gx, ox, fl.G, fl.L);
    const float bx = CULL ? (ox < 0 ? lo2[0] : (ox > 0 ? hi2[0] : 0.0f)) : 0.0f;
    for (int oy = -1; oy <= 1; ++oy) {
      const int cy = wrapCoord(gy + oy, fl.G);
      const float sy = imageShift(gy, oy, fl.G, fl.L);
      const float bxy = CULL ? bx + (oy < 0 ? lo2[1] : (oy > 0 ? hi2[1] : 0.0f)) : 0.0f;
      if (CULL && cull && bxy > cullThr) continue;
      uint32_t st[3], en[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const int cz = wrapCoord(gz + k - 1, fl.G);
        const uint32_t h = fl.cellBase + ((uint32_t)cz * fl.G + (uint32_t)cy) * fl.G + (uint32_t)cx;
        st[k] = __ldg(&cellStart[h]);
        en[k] = __ldg(&cellEnd[h]);
      }
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const uint32_t start = st[k];
        uint32_t stop = en[k];
        if (!usableRange(fl, start, stop)) continue;
        if (CULL && cull && bxy + (k == 0 ? lo2[2] : (k == 2 ? hi2[2] : 0.0f)) > cullThr) continue;
        if (fl.maxPerCell && stop - start > fl.maxPerCell) stop = start + fl.maxPerCell;
        const float sz = imageShift(gz, k - 1, fl.G, fl.L);
        // Without an image shift (every cell away from the periodic seam)
        // (q + 0) - p and q - p differ at most in the sign of a zero, which
        // the squares remove: the cheaper form gives the same d2 bit for bit.
        const bool shifted = sx != 0.0f || sy != 0.0f || sz != 0.0f;
        uint32_t j = start;
        for (; j + UNROLL <= stop; j += UNROLL) {
          float4 q[UNROLL];
#pragma unroll
          for (int u = 0; u < UNROLL; ++u) q[u] = __ldg(&posS[j + u]);
#pragma unroll
          for (int u = 0; u < UNROLL; ++u) {
            const uint32_t jj = j + u;
            float dx, dy, dz;
            if (shifted) {
              dx = (q[u].x + sx) - p.x; dy = (q[u].y + sy) - p.y; dz = (q[u].z + sz) - p.z;
            } else {
              dx = q[u].x - p.x; dy = q[u].y - p.y; dz = q[u].z - p.z;
            }
            const float d2 = dx * dx + dy * dy + dz * dz;
            if (!(d2 > thr) && jj != self) {
              list[(n++) * ls] = jj;
              if (n == M) return n;
            }
          }
        }
        if (j < stop) {
          float4 q[UNROLL];
#pragma unroll
          for (int u = 0; u < UNROLL; ++u)
            q[u] = (j + u < stop) ? __ldg(&posS[j + u]) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
          for (int u = 0; u < UNROLL; ++u) {
            const uint32_t jj = j + u;
            if (jj < stop && jj != self) {
              const float dx = (q[u].x + sx) - p.x, dy = (q[u].y + sy) - p.y, dz = (q[u].z + sz) - p.z;
              const float d2 = dx * dx + dy * dy + dz * dz;
              if (!(d2 > thr)) {
                list[(n++) * ls] = jj;
                if (n == M) return n;
              }
            }
          }
        }
      }
    }
  }
  return n;
}

// Warp-cooperative neighbour lists, one home cell at a time.
//
// All agents of a home cell share the same 27 neighbour cells in the same
// visit order.  The warp's lanes form runs of equal home cell (sorted
// order); for each run the warp lays the 27 cells' candidates out as one
// sequence in the reference's visit order (x outer, y, z inner; ascending
// slot inside a cell), loads 32 consecutive candidates at a time (one per
// lane), and every agent of the run tests the 32 with one instruction
// sequence: a ballot of the accepting lanes and a population count below
// each lane give the position of each accepted candidate in that agent's
// list.  Lists are identical to the per-agent scan: same candidates, same
// order, same predicate !(d2 > r2thr) on ((q + s) - p)^2 sums, self excluded,
// first M kept.  Cells are not culled: every candidate of the 27 cells is
// tested, so a NaN candidate (which passes every agent's test) is never lost.
//
// With R > 0 the run's first R rounds of candidates are loaded into registers
// up front and each agent then goes through them alone (agent-major): its
// position, slot and count are broadcast once instead of once a round, and
// it stops at the round that fills its list.  With WINT > 0 the next R
// rounds go the same way while at least WINT of the run's agents are still
// open; rounds after that go round-major as with R = 0.  Each agent's list
// gets the same candidates in the same order either way.
//
// With CULL, candidates are first tested against the run's bounding box (the
// smallest box holding the run's agents): a candidate whose squared distance
// to the box exceeds the radius threshold fails every agent's test, and is
// dropped before the votes.  The squared box distance is built like an
// agent's d2, (ex * ex + ey * ey) + ez * ez with ex = max(lo - q, q - hi, 0),
// and rounding is monotone, so it is never above any agent's d2: no
// candidate an agent accepts is dropped.  A NaN d2 passes the test, so runs
// holding a non-finite agent coordinate take an unbounded box, and candidates
// with a non-finite coordinate are always kept.  The survivors keep their order in
// a per-warp staging buffer cbuf ((R + 1) * 32 entries: x, y, z with the
// image shift, slot in w) and are voted on R rounds at a time, agent-major.
// The lists are the same as without culling.
//
// Called by all 32 lanes of a warp; `active` lanes own an agent (sorted slot
// `self`, position p, home cell key `key`, flock `flock`).  Each agent's list
// goes to column laneCol0 + lane of the shared array sList (stride ls).
// Returns the lane's list length.
// Rounds of 32 candidates the cooperative scan holds in registers: 96
// candidates cover most home cells' 27-cell neighbourhoods at densities of 3
// to 4 agents a cell (72 to 108 candidates).  Holding 4 measured the same on
// the batched workload and 3% slower on config 1; 2 was slower on both.
constexpr int kCoopCachedRounds = 3;
// The windowed scan (flock kernel scan 5, the Schooling kernel) takes
// further windows while at least this many of a run's agents still need
// candidates (dense cells, e.g. config 1's Gaussian blobs): 4% faster on
// config 1, 1% slower on the uniform batched workload, where runs are short.
// 16 measured between the two.
constexpr int kCoopWindowAgents = 8;

// Position of the (w + 1)-th set bit of m (w < popc(m)): the largest q with
// w or fewer set bits below it.
__device__ __forceinline__ uint32_t nthSetBit(uint32_t m, uint32_t w) {
  uint32_t q = 0;
#pragma unroll
  for (uint32_t step = 16; step > 0; step >>= 1)
    if ((uint32_t)__popc(m & ((1u << (q + step)) - 1u)) <= w) q += step;
  return q;
}

__device__ __forceinline__ uint32_t orderedBits(float x) {
  const uint32_t u = __float_as_uint(x);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float fromOrderedBits(uint32_t u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

// With KNN, runs of a flock with useKnn build the reference's kNN list
// instead (the first M accepted, then each closer candidate replacing the
// entry found farthest, Proximity3D_resources.cu:71-104), still agent-major
// over R register-held rounds: lane k holds entry k of the agent's list and
// its distance (M <= 32), the farthest entry is a warp maximum, and the
// agent's list and distances wait in sList / dList between windows.
//
// The reference's bound is stale: a replacement sets it to the largest
// distance before the replacement, and the new entry may lie above that.  So
// the bound s can rise, but never above the larger of its last two values:
// after a replacement of candidate d (d < s_k) the new bound is
// s_{k+1} = max(list) and the next one is at most max(s_{k+1}, d) <
// max(s_{k+1}, s_k).  A candidate at or beyond B = max(s, previous s) can
// never replace an entry and is skipped before the serial replacements.
// The first M accepted go in with one ballot, as in the first-M scan.
template <int R, int WINT = 0, bool CULL = false, bool KNN = false>
__device__ __forceinline__ uint32_t scanNeighborsCooperative(bool active, uint32_t self, f3 p, uint32_t key,
                                                             const FlockDev* __restrict__ flocks, uint32_t flock,
                                                             const uint32_t* __restrict__ cellStart,
                                                             const uint32_t* __restrict__ cellEnd,
                                                             const float4* __restrict__ posS, uint32_t* sList,
                                                             uint32_t ls, uint32_t laneCol0, float4* cbuf = nullptr,
                                                             float* dList = nullptr) {
  static_assert(!CULL || R > 0, "the culled scan votes on register-held rounds");
  static_assert(!KNN || (R > 0 && !CULL), "the kNN scan votes on register-held rounds, unculled");
  const uint32_t full = 0xFFFFFFFFu;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t myKey = active ? key : 0xFFFFFFFFu;
  const uint32_t prevKey = __shfl_up_sync(full, myKey, 1);
  const bool head = active && (lane == 0 || prevKey != myKey);
  uint32_t heads = __ballot_sync(full, head);
  const uint32_t activeMask = __ballot_sync(full, active);
  uint32_t n = 0;
  float kmx = 0.0f, kmxPrev = 0.0f;  // kNN: the lane's agent's bound (maxDistValue) and its previous value
  // bounding box of the lane's run: lanes of equal key (a run, or with a
  // corrupted order a superset of it, which only culls less)
  float bLo[3] = {0.f, 0.f, 0.f}, bHi[3] = {0.f, 0.f, 0.f};
  if constexpr (CULL) {
    const uint32_t grp = __match_any_sync(full, myKey);
    const uint32_t ox = orderedBits(p.x), oy = orderedBits(p.y), oz = orderedBits(p.z);
    bLo[0] = fromOrderedBits(__reduce_min_sync(grp, ox));
    bLo[1] = fromOrderedBits(__reduce_min_sync(grp, oy));
    bLo[2] = fromOrderedBits(__reduce_min_sync(grp, oz));
    bHi[0] = fromOrderedBits(__reduce_max_sync(grp, ox));
    bHi[1] = fromOrderedBits(__reduce_max_sync(grp, oy));
    bHi[2] = fromOrderedBits(__reduce_max_sync(grp, oz));
    // A non-finite coordinate can make an agent's d2 NaN (NaN - q, or
    // inf - inf), and a NaN d2 passes the test: such a run is not culled.
    const bool finite = isfinite(p.x) && isfinite(p.y) && isfinite(p.z);
    if (__reduce_or_sync(grp, finite ? 0u : 1u)) {
      bLo[0] = bLo[1] = bLo[2] = -INFINITY;
      bHi[0] = bHi[1] = bHi[2] = INFINITY;
    }
  }
  while (heads) {
    const uint32_t g0 = __ffs(heads) - 1;
    heads &= heads - 1;
    const uint32_t g1 = heads ? (__ffs(heads) - 1) : 32u;
    // group lanes [g0, g1) among the active ones
    const uint32_t groupMask = activeMask & (((g1 >= 32u) ? full : ((1u << g1) - 1u)) & ~((1u << g0) - 1u));
    const uint32_t f = __shfl_sync(full, flock, g0);
    const FlockDev& fl = flocks[f];
    const uint32_t M = fl.M;
    const float thr = fl.r2thr;
    const uint32_t G = fl.G;
    // home cell coordinates from the group's first agent
    const float px = __shfl_sync(full, p.x, g0), py = __shfl_sync(full, p.y, g0), pz = __shfl_sync(full, p.z, g0);
    const int gx = gridCoord(px, fl), gy = gridCoord(py, fl), gz = gridCoord(pz, fl);
    // lanes 0..26: one neighbour cell each, in visit order
    uint32_t segStart = 0, segLen = 0;
    float sx = 0.0f, sy = 0.0f, sz = 0.0f;
    if (lane < 27u) {
      const int ox = (int)(lane / 9u) - 1, oy = (int)((lane / 3u) % 3u) - 1, oz = (int)(lane % 3u) - 1;
      const int cx = wrapCoord(gx + ox, G), cy = wrapCoord(gy + oy, G), cz = wrapCoord(gz + oz, G);
      const uint32_t h = fl.cellBase + ((uint32_t)cz * G + (uint32_t)cy) * G + (uint32_t)cx;
      const uint32_t st = __ldg(&cellStart[h]), en = __ldg(&cellEnd[h]);
      if (usableRange(fl, st, en)) {
        segStart = st;
        segLen = en - st;
        if (fl.maxPerCell && segLen > fl.maxPerCell) segLen = fl.maxPerCell;
      }
      sx = imageShift(gx, ox, G, fl.L);
      sy = imageShift(gy, oy, G, fl.L);
      sz = imageShift(gz, oz, G, fl.L);
    }
    // exclusive prefix of the segment lengths
    uint32_t incl = segLen;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(full, incl, o);
      if (lane >= (uint32_t)o) incl += v;
    }
    const uint32_t excl = incl - segLen;
    const uint32_t total = __shfl_sync(full, incl, 31);
    uint32_t open = groupMask;  // group agents whose list is not full yet
    uint32_t base0 = 0;
    if constexpr (KNN) {
      if (fl.useKnn) {
        constexpr uint32_t kNoSlot = 0xFFFFFFFFu;
        const float radius = fl.radius;
        for (; base0 < total; base0 += (uint32_t)R * 32u) {
          float cqx[R], cqy[R], cqz[R];
          uint32_t cslot[R];
#pragma unroll
          for (int r = 0; r < R; ++r) {
            cqx[r] = cqy[r] = cqz[r] = 0.0f;
            cslot[r] = kNoSlot;
            if (base0 + (uint32_t)r * 32u < total) {
              const uint32_t t = base0 + (uint32_t)r * 32u + lane;
              uint32_t c = 0;
#pragma unroll
              for (int step = 16; step > 0; step >>= 1) {
                const uint32_t cand = c + (uint32_t)step;
                const uint32_t e = __shfl_sync(full, excl, cand & 31u);
                if (cand < 27u && e <= t) c = cand;
              }
              const uint32_t cStart = __shfl_sync(full, segStart, c), cExcl = __shfl_sync(full, excl, c);
              const float csx = __shfl_sync(full, sx, c), csy = __shfl_sync(full, sy, c), csz = __shfl_sync(full, sz, c);
              if (t < total) {
                cslot[r] = cStart + (t - cExcl);
                const float4 q = __ldg(&posS[cslot[r]]);
                cqx[r] = q.x + csx;
                cqy[r] = q.y + csy;
                cqz[r] = q.z + csz;
              }
            }
          }
          for (uint32_t todo = groupMask; todo; todo &= todo - 1u) {
            const uint32_t a = __ffs(todo) - 1u;
            const float ax = __shfl_sync(full, p.x, a), ay = __shfl_sync(full, p.y, a), az = __shfl_sync(full, p.z, a);
            const uint32_t aSelf = __shfl_sync(full, self, a);
            uint32_t an = __shfl_sync(full, n, a);
            float amx = __shfl_sync(full, kmx, a), amxPrev = __shfl_sync(full, kmxPrev, a);
            uint32_t* col = sList + laneCol0 + a;
            float* dcol = dList + laneCol0 + a;
            const uint32_t below = (1u << lane) - 1u;
            // the agent's list so far: entry `lane` and its distance
            uint32_t ks = 0u;
            float kd = 0.0f;
            if (lane < an) {
              ks = col[lane * ls];
              kd = dcol[lane * ls];
            }
#pragma unroll
            for (int r = 0; r < R; ++r) {
              if (base0 + (uint32_t)r * 32u >= total) break;
              const float dx = cqx[r] - ax, dy = cqy[r] - ay, dz = cqz[r] - az;
              const float dist = sqrtf(dx * dx + dy * dy + dz * dz);
              const bool acc = cslot[r] != kNoSlot && cslot[r] != aSelf && !(dist > radius);
              uint32_t bal = __ballot_sync(full, acc);
              if (an < M) {
                // the fill: accepted candidates in order into entries an, an + 1, ...
                const uint32_t pos = an + (uint32_t)__popc(bal & below);
                const bool fill = acc && pos < M;
                const uint32_t fillers = __ballot_sync(full, fill);
                {
                  // entry lanes an, an + 1, ... pull their new entry from the
                  // lane of the 1st, 2nd, ... candidate taken
                  const uint32_t want = lane - an;  // wraps for lanes below an
                  const bool mine = lane >= an && want < (uint32_t)__popc(fillers);
                  const uint32_t srcLane = mine ? nthSetBit(fillers, want) : 0u;
                  const float cd = __shfl_sync(full, dist, srcLane);
                  const uint32_t cs = __shfl_sync(full, cslot[r], srcLane);
                  if (mine) { ks = cs; kd = cd; }
                }
                // maxDistValue = max over the entries taken, in order (no NaN
                // is ever kept as the bound by the reference's std::max)
                const uint32_t fb = (fill && !isnan(dist)) ? __float_as_uint(dist) : 0u;
                const uint32_t fm = __reduce_max_sync(full, fb);
                if (fillers) amx = fmaxf(amx, __uint_as_float(fm));
                an += (uint32_t)__popc(fillers);
                bal &= ~fillers;
                amxPrev = amx;
              }
              // the rest: candidates below the bound's ceiling, one at a time
              const float ceilB = fmaxf(amx, amxPrev);
              bal &= __ballot_sync(full, dist < ceilB);
              for (; bal; bal &= bal - 1u) {
                const uint32_t src = __ffs(bal) - 1u;
                const float cd = __shfl_sync(full, dist, src);
                const uint32_t cs = __shfl_sync(full, cslot[r], src);
                if (cd < amx) {
                  // the first entry holding the largest distance, as the
                  // reference's scan from entry 0 with a strict < finds it
                  // (a NaN entry 0 stays the pick; other NaN entries never are)
                  const float d0 = __shfl_sync(full, kd, 0);
                  uint32_t idx = 0;
                  float mv = d0;
                  if (!isnan(d0)) {
                    const bool ok = lane < an && !isnan(kd);
                    const uint32_t kb = ok ? __float_as_uint(kd) : 0u;  // distances are >= +0
                    const uint32_t mb = __reduce_max_sync(full, kb);
                    idx = __ffs(__ballot_sync(full, ok && kb == mb)) - 1u;
                    mv = __uint_as_float(mb);
                  }
                  amxPrev = amx;
                  amx = mv;
                  if (lane == idx) { ks = cs; kd = cd; }
                }
              }
            }
            if (lane < an) {
              col[lane * ls] = ks;
              dcol[lane * ls] = kd;
            }
            if (lane == a) { n = an; kmx = amx; kmxPrev = amxPrev; }
          }
        }
        continue;  // the next run
      }
    }
    if constexpr (CULL) {
      constexpr uint32_t kNoSlot = 0xFFFFFFFFu;
      const uint32_t below = (1u << lane) - 1u;
      const float lx = __shfl_sync(full, bLo[0], g0), ly = __shfl_sync(full, bLo[1], g0), lz = __shfl_sync(full, bLo[2], g0);
      const float hx = __shfl_sync(full, bHi[0], g0), hy = __shfl_sync(full, bHi[1], g0), hz = __shfl_sync(full, bHi[2], g0);
      uint32_t raw = 0;       // next candidate of the run's sequence to test against the box
      uint32_t buffered = 0;  // survivors staged in cbuf[0, buffered), in sequence order
      for (;;) {
        // stage survivors until R rounds' worth are buffered (at most
        // R * 32 - 1 + 32 entries: the buffer holds (R + 1) * 32)
        while (buffered < (uint32_t)R * 32u && raw < total) {
          const uint32_t t = raw + lane;
          uint32_t c = 0;
#pragma unroll
          for (int step = 16; step > 0; step >>= 1) {
            const uint32_t cand = c + (uint32_t)step;
            const uint32_t e = __shfl_sync(full, excl, cand & 31u);
            if (cand < 27u && e <= t) c = cand;
          }
          const uint32_t cStart = __shfl_sync(full, segStart, c), cExcl = __shfl_sync(full, excl, c);
          const float csx = __shfl_sync(full, sx, c), csy = __shfl_sync(full, sy, c), csz = __shfl_sync(full, sz, c);
          bool keep = false;
          float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
          if (t < total) {
            const uint32_t slot = cStart + (t - cExcl);
            const float4 q = __ldg(&posS[slot]);
            v = make_float4(q.x + csx, q.y + csy, q.z + csz, __uint_as_float(slot));
            const float ex = fmaxf(fmaxf(lx - v.x, v.x - hx), 0.0f);
            const float ey = fmaxf(fmaxf(ly - v.y, v.y - hy), 0.0f);
            const float ez = fmaxf(fmaxf(lz - v.z, v.z - hz), 0.0f);
            const float b2 = ex * ex + ey * ey + ez * ez;
            // a candidate with a non-finite coordinate can give a NaN d2,
            // which passes: it is always kept
            keep = !(b2 > thr) || !isfinite(v.x + v.y + v.z);
          }
          const uint32_t bal = __ballot_sync(full, keep);
          if (keep) cbuf[buffered + (uint32_t)__popc(bal & below)] = v;
          buffered += (uint32_t)__popc(bal);
          raw += 32u;
        }
        __syncwarp();
        const uint32_t take = min(buffered, (uint32_t)R * 32u);
        float cqx[R], cqy[R], cqz[R];
        uint32_t cslot[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const uint32_t idx = (uint32_t)r * 32u + lane;
          cqx[r] = cqy[r] = cqz[r] = 0.0f;
          cslot[r] = kNoSlot;
          if (idx < take) {
            const float4 v = cbuf[idx];
            cqx[r] = v.x;
            cqy[r] = v.y;
            cqz[r] = v.z;
            cslot[r] = __float_as_uint(v.w);
          }
        }
        __syncwarp();
        // the (at most 31) survivors past R rounds move to the front; when
        // there are any, take = R * 32 >= 32, so no lane reads an entry
        // another lane writes
        const uint32_t rest = buffered - take;
        if (lane < rest) cbuf[lane] = cbuf[take + lane];
        buffered = rest;
        for (uint32_t todo = open; todo; todo &= todo - 1u) {
          const uint32_t a = __ffs(todo) - 1u;
          const float ax = __shfl_sync(full, p.x, a), ay = __shfl_sync(full, p.y, a), az = __shfl_sync(full, p.z, a);
          const uint32_t aSelf = __shfl_sync(full, self, a);
          uint32_t an = __shfl_sync(full, n, a);
          uint32_t* col = sList + laneCol0 + a;
#pragma unroll
          for (int r = 0; r < R; ++r) {
            if ((uint32_t)r * 32u >= take) break;
            const float dx = cqx[r] - ax, dy = cqy[r] - ay, dz = cqz[r] - az;
            const float d2 = dx * dx + dy * dy + dz * dz;
            const bool acc = cslot[r] != kNoSlot && !(d2 > thr) && cslot[r] != aSelf;
            const uint32_t bal = __ballot_sync(full, acc);
            if (acc) {
              const uint32_t pos = an + (uint32_t)__popc(bal & below);
              if (pos < M) col[pos * ls] = cslot[r];
            }
            an += (uint32_t)__popc(bal);
            if (an >= M) break;
          }
          an = min(an, M);
          if (lane == a) n = an;
          if (an >= M) open &= ~(1u << a);
        }
        __syncwarp();
        if (!open || (raw >= total && buffered == 0)) break;
      }
      continue;  // the next run
    }
    if constexpr (R > 0) {
      constexpr uint32_t kNoSlot = 0xFFFFFFFFu;
      const uint32_t below = (1u << lane) - 1u;
      for (;;) {
        float cqx[R], cqy[R], cqz[R];
        uint32_t cslot[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          cqx[r] = cqy[r] = cqz[r] = 0.0f;
          cslot[r] = kNoSlot;
          if (base0 + (uint32_t)r * 32u < total) {
            const uint32_t t = base0 + (uint32_t)r * 32u + lane;
            uint32_t c = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
              const uint32_t cand = c + (uint32_t)step;
              const uint32_t e = __shfl_sync(full, excl, cand & 31u);
              if (cand < 27u && e <= t) c = cand;
            }
            const uint32_t cStart = __shfl_sync(full, segStart, c), cExcl = __shfl_sync(full, excl, c);
            const float csx = __shfl_sync(full, sx, c), csy = __shfl_sync(full, sy, c), csz = __shfl_sync(full, sz, c);
            if (t < total) {
              cslot[r] = cStart + (t - cExcl);
              const float4 q = __ldg(&posS[cslot[r]]);
              cqx[r] = q.x + csx;
              cqy[r] = q.y + csy;
              cqz[r] = q.z + csz;
            }
          }
        }
        for (uint32_t todo = open; todo; todo &= todo - 1u) {
          const uint32_t a = __ffs(todo) - 1u;
          const float ax = __shfl_sync(full, p.x, a), ay = __shfl_sync(full, p.y, a), az = __shfl_sync(full, p.z, a);
          const uint32_t aSelf = __shfl_sync(full, self, a);
          uint32_t an = __shfl_sync(full, n, a);
          uint32_t* col = sList + laneCol0 + a;
#pragma unroll
          for (int r = 0; r < R; ++r) {
            if (base0 + (uint32_t)r * 32u >= total) break;
            const float dx = cqx[r] - ax, dy = cqy[r] - ay, dz = cqz[r] - az;
            const float d2 = dx * dx + dy * dy + dz * dz;
            const bool acc = cslot[r] != kNoSlot && !(d2 > thr) && cslot[r] != aSelf;
            const uint32_t bal = __ballot_sync(full, acc);
            if (acc) {
              const uint32_t pos = an + (uint32_t)__popc(bal & below);
              if (pos < M) col[pos * ls] = cslot[r];
            }
            an += (uint32_t)__popc(bal);
            if (an >= M) break;
          }
          an = min(an, M);
          if (lane == a) n = an;
          if (an >= M) open &= ~(1u << a);
        }
        base0 += (uint32_t)R * 32u;
        if (WINT == 0 || base0 >= total || __popc(open) < WINT) break;
      }
    }
    for (uint32_t base = base0; base < total && open; base += 32u) {
      const uint32_t t = base + lane;
      const bool valid = t < total;
      // segment of t: the last segment whose exclusive prefix is <= t
      uint32_t c = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const uint32_t cand = c + (uint32_t)step;
        const uint32_t e = __shfl_sync(full, excl, cand & 31u);
        if (cand < 27u && e <= t) c = cand;
      }
      const uint32_t cStart = __shfl_sync(full, segStart, c), cExcl = __shfl_sync(full, excl, c);
      const float csx = __shfl_sync(full, sx, c), csy = __shfl_sync(full, sy, c), csz = __shfl_sync(full, sz, c);
      const uint32_t slot = valid ? cStart + (t - cExcl) : 0xFFFFFFFFu;
      const float4 q = valid ? __ldg(&posS[slot]) : make_float4(0.f, 0.f, 0.f, 0.f);
      const float qx = q.x + csx, qy = q.y + csy, qz = q.z + csz;
      for (uint32_t todo = open; todo; todo &= todo - 1u) {
        const uint32_t a = __ffs(todo) - 1u;
        const float ax = __shfl_sync(full, p.x, a), ay = __shfl_sync(full, p.y, a), az = __shfl_sync(full, p.z, a);
        const uint32_t aSelf = __shfl_sync(full, self, a);
        const uint32_t an = __shfl_sync(full, n, a);
        const float dx = qx - ax, dy = qy - ay, dz = qz - az;
        const float d2 = dx * dx + dy * dy + dz * dz;
        const bool acc = valid && !(d2 > thr) && slot != aSelf;
        const uint32_t bal = __ballot_sync(full, acc);
        if (acc) {
          const uint32_t pos = an + (uint32_t)__popc(bal & ((1u << lane) - 1u));
          if (pos < M) sList[pos * ls + laneCol0 + a] = slot;
        }
        const uint32_t nn = min(M, an + (uint32_t)__popc(bal));
        if (lane == a) n = nn;
        if (nn >= M) open &= ~(1u << a);
      }
    }
  }
  // list entries were written by other lanes of the warp
  __syncwarp();
  return n;
}

// Home-agent context for the steering stages.
struct AgentCtx {
  f3 pos, fwd;
  float speed;
  int g[3];
  bool interior;  // no neighbour can need an image shift
};

__device__ __forceinline__ AgentCtx makeCtx(float4 p4, float4 w4, const FlockDev& fl) {
  AgentCtx a;
  a.pos = xyz(p4);
  a.fwd = xyz(w4);
  a.speed = w4.w;
  a.g[0] = gridCoord(a.pos.x, fl);
  a.g[1] = gridCoord(a.pos.y, fl);
  a.g[2] = gridCoord(a.pos.z, fl);
  const int hi = (int)fl.G - 1;
  a.interior = a.g[0] > 0 && a.g[0] < hi && a.g[1] > 0 && a.g[1] < hi && a.g[2] > 0 && a.g[2] < hi;
  return a;
}

__device__ __forceinline__ f3 neighborImage(const AgentCtx& a, float4 q4, const FlockDev& fl) {
  f3 q = xyz(q4);
  float sx = 0.0f, sy = 0.0f, sz = 0.0f;
  if (!a.interior) {
    sx = imageShiftCells(a.g[0], gridCoord(q.x, fl), fl.G, fl.L);
    sy = imageShiftCells(a.g[1], gridCoord(q.y, fl), fl.G, fl.L);
    sz = imageShiftCells(a.g[2], gridCoord(q.z, fl), fl.G, fl.L);
  }
  return mk3(q.x + sx, q.y + sy, q.z + sz);
}

// inBoidNeighborhood (OpenSteerWrapper_resources.cu:67-92) given the shared
// distance and cosine of the offset.
__device__ __forceinline__ bool inBoid(float dist, float cosAngle, float minR, float maxR, float cosMax) {
  if (dist < minR) return true;
  if (dist > maxR) return false;
  return cosAngle > cosMax;
}

// Separation, alignment and cohesion sums over the list in one pass; each sum
// keeps the sequential order of its own reference loop
// (calcSeparation :166-211, calcAlignment :253-290, calcCohesion :216-249),
// and the results are blended in the flocking demo's order
// (BehaveRT_Flocking.cpp:183-193): steer = ((0 + sep*w) + ali*w) + coh*w.
__device__ __forceinline__ f3 flockingSteer(const AgentCtx& a, const FlockDev& fl, const uint32_t* list, uint32_t ls,
                                            uint32_t n, const float4* __restrict__ posS, const float4* __restrict__ fwdS,
                                            f3 steer, bool SEP, bool ALI, bool COH) {
  f3 sSep = mk3(0.f, 0.f, 0.f), sAli = mk3(0.f, 0.f, 0.f), sCoh = mk3(0.f, 0.f, 0.f);
  uint32_t cSep = 0, cAli = 0, cCoh = 0;
  for (uint32_t k = 0; k < n; ++k) {
    const uint32_t j = list[k * ls];
    const f3 other = neighborImage(a, __ldg(&posS[j]), fl);
    const f3 offset = sub3(other, a.pos);
    const float d2 = dot3(offset, offset);
    const float dist = sqrtf(d2);
    const f3 nrm = mul3(offset, 1.0f / dist);
    const float cosAngle = dot3(a.fwd, nrm);
    if (SEP && inBoid(dist, cosAngle, fl.minR, fl.sep[1], fl.sep[2])) {
      sSep = add3(sSep, div3(offset, -d2));
      ++cSep;
    }
    if (ALI && inBoid(dist, cosAngle, fl.minR, fl.ali[1], fl.ali[2])) {
      sAli = add3(sAli, xyz(__ldg(&fwdS[j])));
      ++cAli;
    }
    if (COH && inBoid(dist, cosAngle, fl.minR, fl.coh[1], fl.coh[2])) {
      sCoh = add3(sCoh, other);
      ++cCoh;
    }
  }
  if (SEP) {
    if (cSep > 0) sSep = normalize3(div3(sSep, (float)cSep));
    steer = add3(mul3(sSep, fl.sep[0]), steer);
  }
  if (ALI) {
    if (cAli > 0) sAli = normalize3(sub3(div3(sAli, (float)cAli), a.fwd));
    steer = add3(mul3(sAli, fl.ali[0]), steer);
  }
  if (COH) {
    if (cCoh > 0) sCoh = normalize3(sub3(div3(sCoh, (float)cCoh), a.pos));
    steer = add3(mul3(sCoh, fl.coh[0]), steer);
  }
  return steer;
}

// calcSeparation alone (OpenSteerWrapper_resources.cu:166-211): the
// normalised mean of -offset / |offset|^2 over the listed neighbours inside
// the separation neighbourhood, zero when there is none.  The per-neighbour
// operations are those of flockingSteer's separation sum.
__device__ __forceinline__ f3 separationDir(const AgentCtx& a, const FlockDev& fl, const uint32_t* list, uint32_t ls,
                                            uint32_t n, const float4* __restrict__ posS) {
  f3 s = mk3(0.f, 0.f, 0.f);
  uint32_t c = 0;
  for (uint32_t k = 0; k < n; ++k) {
    const f3 other = neighborImage(a, __ldg(&posS[list[k * ls]]), fl);
    const f3 offset = sub3(other, a.pos);
    const float d2 = dot3(offset, offset);
    const float dist = sqrtf(d2);
    const f3 nrm = mul3(offset, 1.0f / dist);
    const float cosAngle = dot3(a.fwd, nrm);
    if (inBoid(dist, cosAngle, fl.minR, fl.sep[1], fl.sep[2])) {
      s = add3(s, div3(offset, -d2));
      ++c;
    }
  }
  if (c > 0) s = normalize3(div3(s, (float)c));
  return s;
}

// steerToAvoidNeighbors (OpenSteerWrapper_kernel.cu:110-154): the weighted
// separation force, multiplied by (n - 16) * 0.5 when more than 16 neighbours
// are listed, and the agent's speed scaled by 0.9 when the force points
// against its heading (dot < -0.8) or by 1.02 when along it (dot > 0.5).  The
// thresholds and factors are double literals in the reference, so the
// comparison and the scaling are done in double.  Returns the force; *speed
// is updated in place.
__device__ __forceinline__ f3 avoidNeighbors(const AgentCtx& a, const FlockDev& fl, const uint32_t* list, uint32_t ls,
                                             uint32_t n, const float4* __restrict__ posS, float* speed) {
  f3 s = mul3(separationDir(a, fl, list, ls, n, posS), fl.sep[0]);
  if (n > 16u) s = mul3(s, (float)(n - 16u) * 0.5f);
  const double d = (double)dot3(s, a.fwd);
  if (d < -0.8) *speed = (float)((double)*speed * 0.9);
  else if (d > 0.5) *speed = (float)((double)*speed * 1.02);
  return s;
}

// computeSimilarity (BehaviorClustering_resources.cu:156-180); the self norm
// is the same for every pair and is passed in.
__device__ __forceinline__ float similarity(const float* fi, float norm1, const float* __restrict__ fj, uint32_t F) {
  float dot = 0.0f, n2 = 0.0f;
  for (uint32_t k = 0; k < F; ++k) {
    const float b = __ldg(&fj[k]);
    dot += fi[k] * b;
    n2 += b * b;
  }
  n2 = sqrtf(n2);
  const float s = dot / (norm1 * n2);
  return (s + 1.0f) / 2.0f;
}
__device__ __forceinline__ float selfNorm(const float* fi, uint32_t F) {
  float n1 = 0.0f;
  for (uint32_t k = 0; k < F; ++k) n1 += fi[k] * fi[k];
  return sqrtf(n1);
}

// BehaviorClustering_resources.cu:61-147
__device__ __forceinline__ float linInterp(float x, float xa, float ya, float xb, float yb) {
  return ya * ((x - xb) / (xa - xb)) + yb * ((x - xa) / (xb - xa));
}
__device__ __forceinline__ float interpolateSimilarity(float val, float mn, float avg, float mx) {
  if (val > avg) return clampf(linInterp(val, avg, 0.5f, mx, 1.0f), 0.0f, 1.0f);
  return clampf(linInterp(val, mn, 0.0f, avg, 0.5f), 0.0f, 1.0f);
}
__device__ __forceinline__ float4 updateSimilarityStats(float sim, float4 st, const FlockDev& fl) {
  float minVal = st.x, avgVal = st.y, maxVal = st.z;
  const float ctl = fl.avgCtl;
  const float blend = sim * ctl + ((maxVal + minVal) / 2.0f) * (1.0f - ctl);
  avgVal += (blend - st.y) * fl.simStats[0];
  avgVal = clampf(avgVal, 0.0f, 1.0f);
  if (sim < minVal) {
    minVal += (sim - minVal) * fl.simStats[1];
    if (minVal > avgVal) minVal = clampf(minVal, 0.0f, sim);
  } else if (minVal < avgVal) {
    minVal += fl.simStats[2];
  }
  if (sim > maxVal) {
    maxVal += (sim - maxVal) * fl.simStats[1];
    if (maxVal < avgVal) maxVal = clampf(maxVal, sim, 1.0f);
  } else if (maxVal > avgVal) {
    maxVal -= fl.simStats[2];
  }
  st.x = minVal; st.y = avgVal; st.z = maxVal;
  return st;
}

// xxxsteerForSeek / xxxsteerForFlee (OpenSteerWrapper_resources.cu:294-322)
__device__ __forceinline__ f3 truncateLength(f3 v, float maxLength) {
  const float len = len3(v);
  if (len <= maxLength) return v;
  return mul3(v, maxLength / len);
}

// BehaviorClustering split path (BehaviorClustering_kernel.cu:306-497,
// BehaviorClustering_resources.cu:269-384): adaptive similarity per
// neighbour, then cluster cohesion (seek/flee blend) and cluster alignment,
// each blended into the steering force.  Similarities are staged in `sims`.
__device__ __forceinline__ f3 clusteringSteer(const AgentCtx& a, const FlockDev& fl, const uint32_t* list, uint32_t ls, uint32_t n,
                                              const float4* __restrict__ posS, const float4* __restrict__ fwdS,
                                              const float* fi, float norm1, const float* __restrict__ featS,
                                              uint32_t Fs, float4& stats, float* sims, f3 steer) {
  const bool coh = fl.clus != 0.0f, ali = fl.aclus != 0.0f;
  for (uint32_t k = 0; k < n; ++k) {
    const float s = similarity(fi, norm1, featS + (size_t)list[k * ls] * Fs, fl.F);
    stats = updateSimilarityStats(s, stats, fl);
    sims[k] = interpolateSimilarity(s, stats.x, stats.y, stats.z);
  }
  if (coh) {
    f3 s = mk3(0.f, 0.f, 0.f);
    const f3 myVel = mul3(a.fwd, a.speed);
    for (uint32_t k = 0; k < n; ++k) {
      const float sim = sims[k];
      const f3 other = neighborImage(a, __ldg(&posS[list[k * ls]]), fl);
      const f3 seek = sub3(truncateLength(sub3(other, a.pos), fl.maxSpeed), myVel);
      const f3 flee = sub3(truncateLength(sub3(a.pos, other), fl.maxSpeed), myVel);
      const float om = 1.0f - sim;
      s = add3(s, add3(mul3(seek, sim), mul3(flee, om)));
    }
    if (n > 0) s = mul3(normalize3(div3(s, (float)n)), fl.clus);
    steer = add3(s, steer);
  }
  if (ali) {
    f3 s = mk3(0.f, 0.f, 0.f);
    for (uint32_t k = 0; k < n; ++k) s = add3(s, mul3(xyz(__ldg(&fwdS[list[k * ls]])), sims[k]));
    if (n > 0) s = mul3(normalize3(sub3(div3(s, (float)n), a.fwd)), fl.aclus);
    steer = add3(s, steer);
  }
  return steer;
}

// Bits of the obstacles (by index within the flock) that can reach the
// agent's cell: the per-cell obstacle field built on the grid by the host
// (a superset of the obstacles with d < reach for any position in the cell),
// or every obstacle when the engine has no field.
__device__ __forceinline__ uint64_t obstacleBits(const AgentCtx& a, const FlockDev& fl, const uint2* __restrict__ obsMask) {
  if (obsMask) {
    const uint2 m = __ldg(&obsMask[fl.cellBase + ((uint32_t)a.g[2] * fl.G + (uint32_t)a.g[1]) * fl.G + (uint32_t)a.g[0]]);
    return ((uint64_t)m.y << 32) | m.x;
  }
  return fl.numObstacles >= 64 ? ~0ull : ((1ull << fl.numObstacles) - 1ull);
}

// Static sphere obstacles: flee every sphere whose centre is closer than
// radius + commonSearchRadius, linear falloff to zero there, weight
// obstacleAvoidanceWeight (no reference counterpart; nearest analogue
// moveAwayFromTarget_kernel, OpenSteerWrapper_kernel.cu:185-212).  The
// obstacles are visited in index order; the ones the cell's field leaves
// out contribute nothing, so the sum is the same as over all of them.
__device__ __forceinline__ f3 obstacleSteer(const AgentCtx& a, const FlockDev& fl, const float4* __restrict__ obstacles,
                                            const uint2* __restrict__ obsMask, f3 steer) {
  f3 s = mk3(0.f, 0.f, 0.f);
  const float L = fl.L, hL = 0.5f * fl.L;
  for (uint64_t bits = obstacleBits(a, fl, obsMask); bits; bits &= bits - 1ull) {
    const uint32_t o = (uint32_t)__ffsll((long long)bits) - 1u;
    const float4 c = __ldg(&obstacles[fl.obsBase + o]);
    f3 off = sub3(a.pos, xyz(c));
    if (off.x > hL) off.x = off.x - L; else if (off.x < -hL) off.x = off.x + L;
    if (off.y > hL) off.y = off.y - L; else if (off.y < -hL) off.y = off.y + L;
    if (off.z > hL) off.z = off.z - L; else if (off.z < -hL) off.z = off.z + L;
    const float d = len3(off);
    const float reach = c.w + fl.radius;
    if (d < reach && d > 0.0f) {
      const float t = 1.0f - d / reach;
      s = add3(s, mul3(off, t / d));
    }
  }
  return add3(mul3(s, fl.obsW), steer);
}

// Feature relaxation toward the similarity-weighted neighbour mean (no
// reference counterpart; the similarity is the reference's computeSimilarity).
__device__ __forceinline__ void relaxFeatures(const FlockDev& fl, const uint32_t* list, uint32_t ls, uint32_t n, const float* fi,
                                              float norm1, const float* __restrict__ featS, uint32_t Fs, float* fo) {
  for (uint32_t k = 0; k < fl.F; ++k) fo[k] = fi[k];
  if (fl.relax == 0.0f || fl.F == 0 || n == 0) return;
  float acc[BRT_MAX_FEATUREDIM];
  float sumS = 0.0f;
  for (uint32_t k = 0; k < fl.F; ++k) acc[k] = 0.0f;
  for (uint32_t m = 0; m < n; ++m) {
    const float* fj = featS + (size_t)list[m * ls] * Fs;
    const float s = similarity(fi, norm1, fj, fl.F);
    sumS += s;
    for (uint32_t k = 0; k < fl.F; ++k) acc[k] += s * __ldg(&fj[k]);
  }
  if (sumS > 0.0f) {
    for (uint32_t k = 0; k < fl.F; ++k) {
      const float mean = acc[k] / sumS;
      fo[k] = fi[k] + fl.relax * (mean - fi[k]);
    }
  }
}

// genericApplySteeringForceD / applySteeringForceSingle
// (OpenSteerWrapper_kernel.cu:265-333, OpenSteerWrapper_resources.cu:326-379,
// Core/common_resources.cu:158-271), then wrap into [0, L).
struct Integrated {
  float4 pos, fwd, acc;
};
__device__ __forceinline__ f3 vecLimitDeviationAngle(f3 source, float cosineOfConeAngle, f3 basis) {
  const float sourceLength = len3(source);
  if (sourceLength == 0.0f) return source;
  const f3 direction = div3(source, sourceLength);
  const float cosineOfSourceAngle = dot3(direction, basis);
  if (cosineOfSourceAngle >= cosineOfConeAngle) return source;
  const float projection = dot3(source, basis);
  const f3 perp = sub3(source, mul3(basis, projection));
  const f3 unitPerp = normalize3(perp);
  const float perpDist = sqrtf(1.0f - (cosineOfConeAngle * cosineOfConeAngle));
  const f3 c0 = mul3(basis, cosineOfConeAngle);
  const f3 c1 = mul3(unitPerp, perpDist);
  return mul3(add3(c0, c1), sourceLength);
}
// range^20 of adjustRawSteeringForce's low-speed branch, where the reference
// calls powf(range, 20) (Core/common_resources.cu:251).  Evaluated in double
// by repeated squaring (x^16 * x^4) and rounded to float once.  The CPU
// oracle runs the same operation sequence, so host and device agree bit for
// bit, and the result is the correctly rounded x^20 unless the exact value
// lies within about 6e-16 (relative) of a float rounding boundary.
__host__ __device__ __forceinline__ float pow20f(float x) {
  const double d = (double)x, d2 = d * d, d4 = d2 * d2, d8 = d4 * d4, d16 = d8 * d8;
  return (float)(d16 * d4);
}
// x^19 in the same way (the derivative of pow20f in the adjoint).
__host__ __device__ __forceinline__ float pow19f(float x) {
  const double d = (double)x, d2 = d * d, d4 = d2 * d2, d8 = d4 * d4, d16 = d8 * d8;
  return (float)((d16 * d2) * d);
}
__device__ __forceinline__ f3 adjustRawSteeringForce(f3 force, float speed, f3 forward, float maxSpeed) {
  const float maxAdjustedSpeed = 0.2f * maxSpeed;
  if ((speed > maxAdjustedSpeed) || (force.x == 0.0f && force.y == 0.0f && force.z == 0.0f)) return force;
  const float range = speed / maxAdjustedSpeed;
  const float p = pow20f(range);
  const float cosine = 1.0f + ((-1.0f - 1.0f) * p);
  return vecLimitDeviationAngle(force, cosine, forward);
}
__device__ __forceinline__ float wrapPeriodic(float x, float L) {
  if (x >= L) return x - L;
  if (x < 0.0f) {
    x = x + L;
    if (x >= L) x = 0.0f;
  }
  return x;
}
__device__ __forceinline__ Integrated integrate(const AgentCtx& a, float4 acc4, f3 steer, float dt, const FlockDev& fl) {
  Integrated r;
  if (a.speed < 0.0f) {
    // The agent does not move; the reference writes the steering force into
    // forward (OpenSteerWrapper_kernel.cu:286-294).
    r.pos = make_float4(a.pos.x, a.pos.y, a.pos.z, 1.0f);
    r.acc = acc4;
    r.fwd = make_float4(steer.x, steer.y, steer.z, 0.0f);
    return r;
  }
  f3 force = steer;
  if (fl.use2D) force.y = 0.0f;
  f3 position = a.pos, forward = a.fwd, smoothed = xyz(acc4);
  float speed = a.speed;
  const f3 adjusted = adjustRawSteeringForce(force, speed, forward, fl.maxSpeed);
  const f3 clipped = truncateLength(adjusted, fl.maxForce);
  const f3 newAccel = div3(clipped, fl.mass);
  if (dt > 0.0f) {
    const float smoothRate = clampf(9.0f * dt, 0.15f, 0.4f);
    const float alpha = clampf(smoothRate, 0.0f, 1.0f);
    smoothed = add3(smoothed, mul3(sub3(newAccel, smoothed), alpha));
  }
  f3 v = add3(mul3(forward, speed), mul3(smoothed, dt));
  v = truncateLength(v, fl.maxSpeed);
  speed = len3(v);
  position = add3(position, mul3(v, dt));
  if (fl.use2D) v.y = 0.0f;
  forward = normalize3(v);
  if (fl.use2D) position.y = 0.5f;
  r.pos = make_float4(wrapPeriodic(position.x, fl.L), wrapPeriodic(position.y, fl.L), wrapPeriodic(position.z, fl.L), 1.0f);
  r.acc = make_float4(smoothed.x, smoothed.y, smoothed.z, acc4.w);
  r.fwd = make_float4(forward.x, forward.y, forward.z, speed);
  return r;
}

}  // namespace brt
