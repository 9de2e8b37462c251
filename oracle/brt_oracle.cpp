// brt_oracle.cpp -- CPU oracle of BehaveRT's per-step agent pipeline.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, in plain C++, the algorithm
// of the reference's per-step pipeline so that the CUDA path can be checked
// against it.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline / reference arm may load it; the product library never does.
//
// Parity pinning: the reference ships no tests, fixtures or golden vectors
// for this path, and its CUDA build cannot run here (cutil, texture
// references, GL interop, MSVC-only constructs).  Its device functions and
// per-agent kernels of this path do compile on the host with small
// stand-ins (oracle/build_ref.py, oracle/ref_shim/): cell hash, neighbour
// search in visit order with the maxNeighbors cap (first-M and kNN),
// inBoidNeighborhood, separation / alignment / cohesion, adjustRawSteeringForce
// and applySteeringForceSingle, and one whole frame of the flocking demo
// through genericCalcNeighgborhoodD, genericSeparationD / AlignmentD /
// CohesionD and genericApplySteeringForceD.  tests/test_oracle_reference.py
// checks this restatement against them bit for bit.  Each function cites the
// reference lines it follows.
//
// Two modes share one template:
//   mode 0 (FP32): float arithmetic in the reference's operation order, built
//                  with -ffp-contract=off so every + - * / sqrt is one IEEE
//                  rounding (the CUDA kernels are built with --fmad=false);
//   mode 1 (FP64): the same operation sequence in double.  Cell hashes, the
//                  sort and neighbour lists always use the FP32 predicate on
//                  float-rounded positions ("frozen" neighbour sets), so the
//                  FP64 result isolates floating-point error of the forces,
//                  integration and feature update.
//
// Deliberate, documented deltas from the reference (shared with the CUDA path):
//   * periodic cube [0, L)^3 with origin 0 instead of the padded clamped box;
//     neighbour cells wrap, and a neighbour reached through a wrap is used at
//     its image position q + s, s in {-L, 0, +L} per axis (computed in the
//     working precision);
//   * cellStart and cellEnd (empty = 0xFFFFFFFF) instead of cellStart only;
//   * neighbour lists are read at the stride they are written (M+1), not at
//     the reference's uint4 word stride (Proximity3D_resources.cu:175-198);
//   * normalize(v) = v * (1 / sqrt(dot(v, v))) (cutil's host form);
//   * positions are wrapped back into [0, L) after integration;
//   * the neighbour scan stops once maxNeighbors entries are held and kNN is
//     off (the remaining candidates cannot change the list).
#include "../include/behavert_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;

template <class R> struct V3 { R x, y, z; };
template <class R> inline V3<R> mk(R x, R y, R z) { return V3<R>{x, y, z}; }
template <class R> inline V3<R> operator+(V3<R> a, V3<R> b) { return mk<R>(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class R> inline V3<R> operator-(V3<R> a, V3<R> b) { return mk<R>(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class R> inline V3<R> operator*(V3<R> a, R s) { return mk<R>(a.x * s, a.y * s, a.z * s); }
template <class R> inline V3<R> operator/(V3<R> a, R s) { return mk<R>(a.x / s, a.y / s, a.z / s); }
template <class R> inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline R length(V3<R> a) { return std::sqrt(dot(a, a)); }
// cutil_math normalize with the host rsqrtf = 1/sqrtf.
template <class R> inline V3<R> normalize(V3<R> v) { R inv = R(1) / std::sqrt(dot(v, v)); return v * inv; }
template <class R> inline R clampf(R f, R a, R b) { return std::fmax(a, std::fmin(f, b)); }
// x^20 of adjustRawSteeringForce's low-speed branch (the reference's
// powf(range, 20), Core/common_resources.cu:251).  FP32 mode: computed in
// double by repeated squaring (x^16 * x^4) and rounded to float once, the
// operation sequence of the CUDA library's pow20f (the reference's powf is a
// library routine whose last bit differs between CUDA and glibc; this form is
// the correctly rounded power unless the exact value lies within ~6e-16 of a
// float rounding boundary, and is the same on both sides).  FP64 mode: pow.
inline float pow20(float x) {
  const double d = (double)x, d2 = d * d, d4 = d2 * d2, d8 = d4 * d4, d16 = d8 * d8;
  return (float)(d16 * d4);
}
inline double pow20(double x) { return std::pow(x, 20.0); }

// Core/common_resources.cu:140-143
template <class R> inline R interpolate(R alpha, R x0, R x1) { return x0 + ((x1 - x0) * alpha); }
template <class R> inline V3<R> interpolate3(R alpha, V3<R> x0, V3<R> x1) { return x0 + ((x1 - x0) * alpha); }

// Core/common_resources.cu:260-271
template <class R> inline V3<R> truncateLength(V3<R> v, R maxLength) {
  R len = length(v);
  if (len <= maxLength) return v;
  return v * (maxLength / len);
}

// Core/common_resources.cu:117-133
template <class R> inline V3<R> perpendicularComponent(V3<R> v, V3<R> unitBasis) {
  R projection = dot(v, unitBasis);
  return v - unitBasis * projection;
}

// Core/common_resources.cu:186-228 (insideOrOutside == true)
template <class R> V3<R> vecLimitDeviationAngleUtility(V3<R> source, R cosineOfConeAngle, V3<R> basis) {
  R sourceLength = length(source);
  if (sourceLength == 0) return source;
  V3<R> direction = source / sourceLength;
  R cosineOfSourceAngle = dot(direction, basis);
  if (cosineOfSourceAngle >= cosineOfConeAngle) return source;
  V3<R> perp = perpendicularComponent(source, basis);
  V3<R> unitPerp = normalize(perp);
  R perpDist = std::sqrt(R(1) - (cosineOfConeAngle * cosineOfConeAngle));
  V3<R> c0 = basis * cosineOfConeAngle;
  V3<R> c1 = unitPerp * perpDist;
  return (c0 + c1) * sourceLength;
}

// Core/common_resources.cu:234-254
template <class R> V3<R> adjustRawSteeringForce(V3<R> force, R speed, V3<R> forward, R maxSpeed) {
  R maxAdjustedSpeed = R(0.2f) * maxSpeed;
  if ((speed > maxAdjustedSpeed) || (force.x == 0 && force.y == 0 && force.z == 0)) return force;
  R range = speed / maxAdjustedSpeed;
  R cosine = interpolate(pow20(range), R(1), R(-1));
  return vecLimitDeviationAngleUtility(force, cosine, forward);
}

// OpenSteerWrapper_resources.cu:67-92
template <class R> bool inBoidNeighborhood(V3<R> myPos, V3<R> otherPos, R minDist, R maxDist, R cosMaxAngle, V3<R> forward) {
  V3<R> offset = otherPos - myPos;
  R dist = length(offset);
  if (dist < minDist) return true;
  if (dist > maxDist) return false;
  R cosAngle = dot(forward, normalize(offset));
  return cosAngle > cosMaxAngle;
}

// OpenSteerWrapper_resources.cu:294-322
template <class R> V3<R> steerForSeek(V3<R> myPos, R mySpeed, V3<R> myForward, V3<R> target, R maxSpeed) {
  V3<R> offset = target - myPos;
  V3<R> desired = truncateLength(offset, maxSpeed);
  V3<R> myVel = myForward * mySpeed;
  return desired - myVel;
}
template <class R> V3<R> steerForFlee(V3<R> myPos, R mySpeed, V3<R> myForward, V3<R> target, R maxSpeed) {
  V3<R> offset = myPos - target;
  V3<R> desired = truncateLength(offset, maxSpeed);
  V3<R> myVel = myForward * mySpeed;
  return desired - myVel;
}

// BehaviorClustering_resources.cu:156-180
template <class R> R computeSimilarity(const R* f1, const R* f2, uint32_t F) {
  R norma1 = 0, norma2 = 0, dot_scalar = 0;
  for (uint32_t k = 0; k < F; ++k) {
    R a = f1[k], b = f2[k];
    dot_scalar += (a * b);
    norma1 += (a * a);
    norma2 += (b * b);
  }
  norma1 = std::sqrt(norma1);
  norma2 = std::sqrt(norma2);
  R similarity = dot_scalar / (norma1 * norma2);
  return (similarity + R(1)) / R(2);
}

// BehaviorClustering_resources.cu:61-69
template <class R> R getLinearInterpolation(R x, R xa, R ya, R xb, R yb) {
  return ya * ((x - xb) / (xa - xb)) + yb * ((x - xa) / (xb - xa));
}
// BehaviorClustering_resources.cu:74-87
template <class R> R interpolateSimilarity(R val, R mn, R avg, R mx) {
  if (val > avg) return clampf(getLinearInterpolation(val, avg, R(0.5f), mx, R(1)), R(0), R(1));
  return clampf(getLinearInterpolation(val, mn, R(0), avg, R(0.5f)), R(0), R(1));
}
// BehaviorClustering_resources.cu:92-147
template <class R> void updateSimilarityStats(R similarity, R st[4], const brt_params& p) {
  R minVal = st[0], avgVal = st[1], maxVal = st[2];
  R ctl = R(p.avgSimilarityController);
  R valueToBlendInAvg = similarity * ctl + ((maxVal + minVal) / R(2)) * (R(1) - ctl);
  avgVal += (valueToBlendInAvg - st[1]) * R(p.similarityStatsParams[0]);
  avgVal = clampf(avgVal, R(0), R(1));
  if (similarity < minVal) {
    minVal += (similarity - minVal) * R(p.similarityStatsParams[1]);
    if (minVal > avgVal) minVal = clampf(minVal, R(0), similarity);
  } else if (minVal < avgVal) {
    minVal += R(p.similarityStatsParams[2]);
  }
  if (similarity > maxVal) {
    maxVal += (similarity - maxVal) * R(p.similarityStatsParams[1]);
    if (maxVal < avgVal) maxVal = clampf(maxVal, similarity, R(1));
  } else if (maxVal > avgVal) {
    maxVal -= R(p.similarityStatsParams[2]);
  }
  st[0] = minVal; st[1] = avgVal; st[2] = maxVal;
}

// Geometry of one flock, derived from its params.
struct Flock {
  brt_params p;
  uint32_t G = 0, C = 0, n = 0;
  uint32_t cellBase = 0, agentBase = 0;
  float L = 0, cell = 0;
};

// envgrid3d_resources.cu:60-84 (calcGridPos + clamping calcGridHash), origin 0.
// calcGridPos assigns floor(...) to an int in device code, a conversion that
// saturates at the int range and takes NaN to 0 (PTX cvt.rzi.s32.f32); a
// plain C++ cast of +inf or of a value past the int range is undefined (x86
// gives INT_MIN, which would clamp to cell 0 instead of G - 1).
inline int deviceFloatToInt(float v) {
  if (std::isnan(v)) return 0;
  if (v >= 2147483648.0f) return INT32_MAX;
  if (v < -2147483648.0f) return INT32_MIN;
  return (int)v;
}
inline int gridCoord(float x, float cell, uint32_t G) {
  int g = deviceFloatToInt(std::floor(x / cell));
  return std::max(0, std::min(g, (int)G - 1));
}
inline uint32_t cellHash(int gx, int gy, int gz, uint32_t G) {
  return ((uint32_t)gz * G + (uint32_t)gy) * G + (uint32_t)gx;
}

// Image shift of a neighbour reached from home coordinate g through offset o.
inline float imageShift(int g, int o, uint32_t G, float L) {
  if (o < 0 && g == 0) return -L;
  if (o > 0 && g == (int)G - 1) return L;
  return 0.0f;
}
inline int wrapCoord(int c, uint32_t G) {
  if (c < 0) return c + (int)G;
  if (c >= (int)G) return c - (int)G;
  return c;
}

template <class R> struct State {
  std::vector<R> pos, fwd, acc, feat, stats;  // sorted order
};

struct Shared {
  std::vector<Flock> fl;
  uint32_t N = 0, Ctot = 0, Mmax = 0, Fmax = 0;
  std::vector<uint32_t> flockOfAgent;  // by agent id
  std::vector<uint32_t> keys;          // by agent id
  std::vector<uint32_t> sortedIds, sortedKeys, cellStart, cellEnd;
  std::vector<float> sposf;            // float sorted positions, 4/agent
  std::vector<uint32_t> lists;         // per sorted slot, stride Mmax+1
  std::vector<uint32_t> scanned;       // candidates examined per sorted slot
};

int setupFlocks(Shared& S, uint32_t nflocks, const brt_params* params) {
  S.fl.resize(nflocks);
  uint32_t cellBase = 0, agentBase = 0;
  S.Mmax = 0; S.Fmax = 0;
  for (uint32_t f = 0; f < nflocks; ++f) {
    Flock& F = S.fl[f];
    F.p = params[f];
    F.L = F.p.worldSize;
    F.cell = F.p.cellSize;
    double g = (double)F.L / (double)F.cell;
    F.G = (uint32_t)std::lround(g);
    if (F.G < 3 || std::fabs(g - F.G) > 1e-6 * g) return BRT_ERR_CONFIG;
    if ((float)F.G * F.cell != F.L) return BRT_ERR_CONFIG;
    if (F.p.maxNeighbors < 1 || F.p.maxNeighbors > BRT_MAX_NEIGHBORS) return BRT_ERR_CONFIG;
    if (F.p.featuresCount > BRT_MAX_FEATUREDIM) return BRT_ERR_CONFIG;
    F.C = F.G * F.G * F.G;
    F.n = F.p.numBodies;
    F.cellBase = cellBase;
    F.agentBase = agentBase;
    cellBase += F.C;
    agentBase += F.n;
    S.Mmax = std::max(S.Mmax, F.p.maxNeighbors);
    S.Fmax = std::max(S.Fmax, F.p.featuresCount);
  }
  S.N = agentBase;
  S.Ctot = cellBase;
  S.flockOfAgent.resize(S.N);
  for (uint32_t f = 0; f < nflocks; ++f)
    for (uint32_t i = 0; i < S.fl[f].n; ++i) S.flockOfAgent[S.fl[f].agentBase + i] = f;
  return BRT_OK;
}

template <class F> void parallelFor(uint32_t n, int threads, F fn) {
  if (threads <= 1 || n < 1024) { fn(0u, n); return; }
  std::vector<std::thread> th;
  uint32_t chunk = (n + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    uint32_t b = t * chunk, e = std::min(n, b + chunk);
    if (b >= e) break;
    th.emplace_back(fn, b, e);
  }
  for (auto& x : th) x.join();
}

// genCalcHashD (envgrid3d_kernel.cu:55-68) + RadixSort semantics
// (radixsort.cu:50-80: stable key/value sort, ties keep input = agent-id order)
// + genericFindCellStartD (Proximity3D_kernel.cu:54-84) extended with cellEnd.
void hashSortRanges(Shared& S, const float* posf /*id order, 4/agent*/) {
  S.keys.resize(S.N);
  for (uint32_t i = 0; i < S.N; ++i) {
    const Flock& F = S.fl[S.flockOfAgent[i]];
    const float* p = posf + 4 * (size_t)i;
    int gx = gridCoord(p[0], F.cell, F.G), gy = gridCoord(p[1], F.cell, F.G), gz = gridCoord(p[2], F.cell, F.G);
    S.keys[i] = F.cellBase + cellHash(gx, gy, gz, F.G);
  }
  // stable counting sort by key
  std::vector<uint32_t> count(S.Ctot + 1, 0);
  for (uint32_t i = 0; i < S.N; ++i) count[S.keys[i] + 1]++;
  for (uint32_t c = 0; c < S.Ctot; ++c) count[c + 1] += count[c];
  S.sortedIds.resize(S.N);
  S.sortedKeys.resize(S.N);
  std::vector<uint32_t> cursor(count.begin(), count.end() - 1);
  for (uint32_t i = 0; i < S.N; ++i) {
    uint32_t k = S.keys[i];
    uint32_t slot = cursor[k]++;
    S.sortedIds[slot] = i;
    S.sortedKeys[slot] = k;
  }
  S.cellStart.assign(S.Ctot, kEmpty);
  S.cellEnd.assign(S.Ctot, kEmpty);
  for (uint32_t s = 0; s < S.N; ++s) {
    uint32_t k = S.sortedKeys[s];
    if (s == 0 || S.sortedKeys[s - 1] != k) S.cellStart[k] = s;
    if (s + 1 == S.N || S.sortedKeys[s + 1] != k) S.cellEnd[k] = s + 1;
  }
  S.sposf.resize(4 * (size_t)S.N);
  for (uint32_t s = 0; s < S.N; ++s)
    std::memcpy(&S.sposf[4 * (size_t)s], posf + 4 * (size_t)S.sortedIds[s], 16);
}

// genericCalcNeighgborhoodD (Proximity3D_kernel.cu:89-125) with
// checkForNeighborsInCell / checkForNeighbor (Proximity3D_resources.cu:59-172),
// periodic version.  Visit order: x outermost, then y, z innermost; within a
// cell ascending sorted slot; self skipped by slot; accept iff
// !(sqrtf(dx*dx+dy*dy+dz*dz) > radius).
void neighborLists(Shared& S, int threads) {
  const uint32_t stride = S.Mmax + 1;
  S.lists.assign((size_t)S.N * stride, 0u);
  S.scanned.assign(S.N, 0u);
  parallelFor(S.N, threads, [&](uint32_t b, uint32_t e) {
    uint32_t list[BRT_MAX_NEIGHBORS];
    float distList[BRT_MAX_NEIGHBORS];
    for (uint32_t i = b; i < e; ++i) {
      const Flock& F = S.fl[S.flockOfAgent[S.sortedIds[i]]];
      const uint32_t M = F.p.maxNeighbors;
      const float r = F.p.commonSearchRadius;
      const bool knn = F.p.useKnn != 0;
      const uint32_t maxPerCell = F.p.maxBodiesPerCell ? F.p.maxBodiesPerCell : 0xFFFFFFFFu;
      const float* p = &S.sposf[4 * (size_t)i];
      int g[3] = {gridCoord(p[0], F.cell, F.G), gridCoord(p[1], F.cell, F.G), gridCoord(p[2], F.cell, F.G)};
      uint32_t n = 0, scanned = 0;
      float maxDistValue = 0.0f;
      bool done = false;
      for (int ox = -1; ox <= 1 && !done; ++ox)
        for (int oy = -1; oy <= 1 && !done; ++oy)
          for (int oz = -1; oz <= 1 && !done; ++oz) {
            int cx = wrapCoord(g[0] + ox, F.G), cy = wrapCoord(g[1] + oy, F.G), cz = wrapCoord(g[2] + oz, F.G);
            float sx = imageShift(g[0], ox, F.G, F.L), sy = imageShift(g[1], oy, F.G, F.L), sz = imageShift(g[2], oz, F.G, F.L);
            uint32_t h = F.cellBase + cellHash(cx, cy, cz, F.G);
            uint32_t start = S.cellStart[h];
            if (start == kEmpty) continue;
            uint32_t end = S.cellEnd[h];
            for (uint32_t t = 0; t < maxPerCell; ++t) {
              uint32_t j = start + t;
              if (j >= end) break;
              if (j == i) continue;
              ++scanned;
              const float* q = &S.sposf[4 * (size_t)j];
              float qx = q[0] + sx, qy = q[1] + sy, qz = q[2] + sz;
              float dx = qx - p[0], dy = qy - p[1], dz = qz - p[2];
              float dist = std::sqrt(dx * dx + dy * dy + dz * dz);
              if (dist > r) continue;
              if (n < M) {
                list[n] = j;
                if (knn) { distList[n] = dist; maxDistValue = std::max(maxDistValue, dist); }
                ++n;
              } else if (knn && dist < maxDistValue) {
                maxDistValue = distList[0];
                uint32_t maxIdx = 0;
                for (uint32_t k = 1; k < n; ++k)
                  if (maxDistValue < distList[k]) { maxDistValue = distList[k]; maxIdx = k; }
                list[maxIdx] = j;
                distList[maxIdx] = dist;
              }
              if (n == M && !knn) { done = true; break; }
            }
          }
      uint32_t* out = &S.lists[(size_t)i * stride];
      out[0] = n;
      for (uint32_t k = 0; k < n; ++k) out[1 + k] = list[k];
      S.scanned[i] = scanned;
    }
  });
}

// Image position of sorted slot j as a neighbour of sorted slot i (same
// convention as the list construction: shift by cell wrap).
template <class R> V3<R> imagePos(const Flock& F, const R* pj, const float* pif, const float* pjf) {
  R s[3];
  for (int a = 0; a < 3; ++a) {
    int gi = gridCoord(pif[a], F.cell, F.G), gj = gridCoord(pjf[a], F.cell, F.G);
    R sh = 0;
    if (gi == 0 && gj == (int)F.G - 1) sh = -R(F.L);
    else if (gi == (int)F.G - 1 && gj == 0) sh = R(F.L);
    s[a] = sh;
  }
  return mk<R>(pj[0] + s[0], pj[1] + s[1], pj[2] + s[2]);
}

template <class R> inline V3<R> v3(const R* a) { return mk<R>(a[0], a[1], a[2]); }

// Per sorted slot: steering stages in the BehaveRT_Clustering update order
// (separation, alignment, cohesion, cluster cohesion, cluster alignment;
// BehaveRT_Clustering.cpp:209-222), obstacle avoidance, then the OpenSteer
// integration (genericApplySteeringForceD, OpenSteerWrapper_kernel.cu:265-333).
template <class R>
void steerIntegrate(const Shared& S, const State<R>& st, R dt, State<R>& out, R* steerOut, bool avoidNeighbors,
                    const float* moveAway, int threads) {
  const uint32_t stride = S.Mmax + 1;
  const uint32_t Fd = S.Fmax;
  parallelFor(S.N, threads, [&](uint32_t b, uint32_t e) {
    std::vector<R> simAd(BRT_MAX_NEIGHBORS);
    std::vector<V3<R>> img(BRT_MAX_NEIGHBORS);
    for (uint32_t i = b; i < e; ++i) {
      const Flock& F = S.fl[S.flockOfAgent[S.sortedIds[i]]];
      const brt_params& p = F.p;
      const uint32_t* lst = &S.lists[(size_t)i * stride];
      const uint32_t n = lst[0];
      const R* P = &st.pos[4 * (size_t)i];
      const R* W = &st.fwd[4 * (size_t)i];
      V3<R> myPos = v3(P), myFwd = v3(W);
      R mySpeed = W[3];
      const float* pif = &S.sposf[4 * (size_t)i];
      for (uint32_t k = 0; k < n; ++k) {
        uint32_t j = lst[1 + k];
        img[k] = imagePos<R>(F, &st.pos[4 * (size_t)j], pif, &S.sposf[4 * (size_t)j]);
      }
      V3<R> steer = mk<R>(0, 0, 0);
      const R minR = R(p.commonSensingMinRadius);
      // The crowd update order replaces computeSeparations by
      // steerAndSlowToAvoidNeighbors (OpenSteerWrapper_kernel.cu:110-154):
      // the weighted separation, times (n - 16) * 0.5f above 16 listed
      // neighbours, and the speed scaled by the double literals 0.9 / 1.02
      // when the force points against / along the heading.  The new speed is
      // what every later stage and the integration read.
      if (avoidNeighbors) {
        V3<R> s = mk<R>(0, 0, 0);
        uint32_t cnt = 0;
        for (uint32_t k = 0; k < n; ++k) {
          if (inBoidNeighborhood(myPos, img[k], minR, R(p.separationParams[1]), R(p.separationParams[2]), myFwd)) {
            V3<R> offset = img[k] - myPos;
            R d2 = dot(offset, offset);
            s = s + offset / (-d2);
            ++cnt;
          }
        }
        if (cnt > 0) s = normalize(s / (R)cnt);
        s = s * R(p.separationParams[0]);
        if (n > 16u) s = s * R((float)(n - 16u) * 0.5f);
        const double d = (double)dot(s, myFwd);
        if (d < -0.8) mySpeed = R((double)mySpeed * 0.9);
        else if (d > 0.5) mySpeed = R((double)mySpeed * 1.02);
        steer = s + steer;
      }
      // calcSeparation (OpenSteerWrapper_resources.cu:166-211), genericSeparationD (:86-105)
      if (!avoidNeighbors && p.separationParams[0] != 0.0f) {
        V3<R> s = mk<R>(0, 0, 0);
        uint32_t cnt = 0;
        for (uint32_t k = 0; k < n; ++k) {
          if (inBoidNeighborhood(myPos, img[k], minR, R(p.separationParams[1]), R(p.separationParams[2]), myFwd)) {
            V3<R> offset = img[k] - myPos;
            R d2 = dot(offset, offset);
            s = s + offset / (-d2);
            ++cnt;
          }
        }
        if (cnt > 0) s = normalize(s / (R)cnt);
        steer = (s * R(p.separationParams[0])) + steer;
      }
      // calcAlignment (:253-290), genericAlignmentD (:158-178)
      if (p.alignmentParams[0] != 0.0f) {
        V3<R> s = mk<R>(0, 0, 0);
        uint32_t cnt = 0;
        for (uint32_t k = 0; k < n; ++k) {
          if (inBoidNeighborhood(myPos, img[k], minR, R(p.alignmentParams[1]), R(p.alignmentParams[2]), myFwd)) {
            s = s + v3(&st.fwd[4 * (size_t)lst[1 + k]]);
            ++cnt;
          }
        }
        if (cnt > 0) s = normalize((s / (R)cnt) - myFwd);
        steer = (s * R(p.alignmentParams[0])) + steer;
      }
      // calcCohesion (:216-249), genericCohesionD (:62-81)
      if (p.cohesionParams[0] != 0.0f) {
        V3<R> s = mk<R>(0, 0, 0);
        uint32_t cnt = 0;
        for (uint32_t k = 0; k < n; ++k) {
          if (inBoidNeighborhood(myPos, img[k], minR, R(p.cohesionParams[1]), R(p.cohesionParams[2]), myFwd)) {
            s = s + img[k];
            ++cnt;
          }
        }
        if (cnt > 0) s = normalize((s / (R)cnt) - myPos);
        steer = (s * R(p.cohesionParams[0])) + steer;
      }
      // BehaviorClustering split path: naive similarities, adaptive stats,
      // cluster cohesion, cluster alignment (BehaviorClustering_kernel.cu:306-497,
      // BehaviorClustering_resources.cu:269-384).
      R stats[4];
      for (int a = 0; a < 4; ++a) stats[a] = st.stats[4 * (size_t)i + a];
      const bool clusCoh = p.clusteringForceParams[0] != 0.0f;
      const bool clusAli = p.alignmentClusteringForceParams[0] != 0.0f;
      const R* fi = Fd ? &st.feat[(size_t)i * Fd] : nullptr;
      if ((clusCoh || clusAli) && p.featuresCount > 0) {
        for (uint32_t k = 0; k < n; ++k) {
          const R* fj = &st.feat[(size_t)lst[1 + k] * Fd];
          R sim = computeSimilarity(fi, fj, p.featuresCount);
          updateSimilarityStats(sim, stats, p);
          simAd[k] = interpolateSimilarity(sim, stats[0], stats[1], stats[2]);
        }
        if (clusCoh) {
          V3<R> s = mk<R>(0, 0, 0);
          R maxSpeed = R(p.commonMaxSpeed);
          for (uint32_t k = 0; k < n; ++k) {
            R sim = simAd[k];
            V3<R> seek = steerForSeek(myPos, mySpeed, myFwd, img[k], maxSpeed);
            V3<R> flee = steerForFlee(myPos, mySpeed, myFwd, img[k], maxSpeed);
            R om = R(1) - sim;
            s = s + ((seek * sim) + (flee * om));
          }
          if (n > 0) s = normalize(s / (R)n) * R(p.clusteringForceParams[0]);
          steer = s + steer;
        }
        if (clusAli) {
          V3<R> s = mk<R>(0, 0, 0);
          for (uint32_t k = 0; k < n; ++k) s = s + v3(&st.fwd[4 * (size_t)lst[1 + k]]) * simAd[k];
          if (n > 0) s = normalize((s / (R)n) - myFwd) * R(p.alignmentClusteringForceParams[0]);
          steer = s + steer;
        }
      }
      // moveAwayFromTarget_kernel (OpenSteerWrapper_kernel.cu:185-212), in the
      // crowd order after cohesion: (w * (p - base)) / |p - base|, zero beyond
      // twice the radius; the direct offset, as in the reference.  Its
      // acceleration write is overwritten by the old value (no effect).
      if (moveAway) {
        V3<R> s = myPos - mk<R>(R(moveAway[0]), R(moveAway[1]), R(moveAway[2]));
        R d = length(s);
        if (d > R(moveAway[5]) * R(2)) s = mk<R>(0, 0, 0);
        steer = ((s * R(moveAway[3])) / d) + steer;
      }
      // Static sphere obstacles: flee every sphere whose centre is closer
      // than radius + commonSearchRadius, with a linear falloff to zero at
      // that distance; weight obstacleAvoidanceWeight.  No reference
      // counterpart (nearest analogue moveAwayFromTarget_kernel).
      if (p.numObstacles > 0 && p.obstacleAvoidanceWeight != 0.0f) {
        V3<R> s = mk<R>(0, 0, 0);
        for (uint32_t o = 0; o < p.numObstacles; ++o) {
          V3<R> c = mk<R>(R(p.obstacles[o][0]), R(p.obstacles[o][1]), R(p.obstacles[o][2]));
          R rad = R(p.obstacles[o][3]);
          V3<R> off = myPos - c;
          // minimum image of the offset in the periodic cube
          R Lr = R(F.L), hL = R(0.5f) * R(F.L);
          if (off.x > hL) off.x = off.x - Lr; else if (off.x < -hL) off.x = off.x + Lr;
          if (off.y > hL) off.y = off.y - Lr; else if (off.y < -hL) off.y = off.y + Lr;
          if (off.z > hL) off.z = off.z - Lr; else if (off.z < -hL) off.z = off.z + Lr;
          R d = length(off);
          R reach = rad + R(p.commonSearchRadius);
          if (d < reach && d > R(0)) {
            R t = R(1) - d / reach;
            s = s + off * (t / d);
          }
        }
        steer = (s * R(p.obstacleAvoidanceWeight)) + steer;
      }
      // computeSeekingsWorldCenter: identity in the periodic cube (every
      // position is inside the world box, OpenSteerWrapper_kernel.cu:236-246).
      if (steerOut) {
        R* so = steerOut + 4 * (size_t)i;
        so[0] = steer.x; so[1] = steer.y; so[2] = steer.z; so[3] = 0;
      }

      // BASELINE feature relaxation toward the similarity-weighted mean.
      R* fo = Fd ? &out.feat[(size_t)i * Fd] : nullptr;
      if (Fd) for (uint32_t a = 0; a < Fd; ++a) fo[a] = fi[a];
      if (p.featureRelaxRate != 0.0f && p.featuresCount > 0 && n > 0) {
        R acc[BRT_MAX_FEATUREDIM];
        R sumS = 0;
        for (uint32_t a = 0; a < p.featuresCount; ++a) acc[a] = 0;
        for (uint32_t k = 0; k < n; ++k) {
          const R* fj = &st.feat[(size_t)lst[1 + k] * Fd];
          R sim = computeSimilarity(fi, fj, p.featuresCount);
          sumS += sim;
          for (uint32_t a = 0; a < p.featuresCount; ++a) acc[a] += sim * fj[a];
        }
        if (sumS > 0) {
          R rate = R(p.featureRelaxRate);
          for (uint32_t a = 0; a < p.featuresCount; ++a) {
            R mean = acc[a] / sumS;
            fo[a] = fi[a] + rate * (mean - fi[a]);
          }
        }
      }
      for (int a = 0; a < 4; ++a) out.stats[4 * (size_t)i + a] = stats[a];

      // genericApplySteeringForceD / applySteeringForceSingle
      // (OpenSteerWrapper_kernel.cu:265-333, OpenSteerWrapper_resources.cu:326-379)
      const R* A = &st.acc[4 * (size_t)i];
      R* po = &out.pos[4 * (size_t)i];
      R* wo = &out.fwd[4 * (size_t)i];
      R* ao = &out.acc[4 * (size_t)i];
      if (mySpeed < 0) {
        // The agent does not move; the reference restores position and
        // acceleration and writes the steering force into forward (:286-294).
        for (int a = 0; a < 3; ++a) po[a] = P[a];
        po[3] = 1;
        for (int a = 0; a < 4; ++a) ao[a] = A[a];
        wo[0] = steer.x; wo[1] = steer.y; wo[2] = steer.z; wo[3] = 0;
        continue;
      }
      V3<R> force = steer;
      if (p.use2DProjection) force.y = 0;
      V3<R> position = myPos, forward = myFwd, smoothedAccel = v3(A);
      R speed = mySpeed;
      R maxSpeed = R(p.commonMaxSpeed);
      V3<R> adjustedForce = adjustRawSteeringForce(force, speed, forward, maxSpeed);
      V3<R> clippedForce = truncateLength(adjustedForce, R(p.commonMaxForce));
      V3<R> newAccel = clippedForce / R(p.commonMass);
      if (dt > 0) {
        R smoothRate = clampf(R(9) * dt, R(0.15f), R(0.4f));
        smoothedAccel = interpolate3(clampf(smoothRate, R(0), R(1)), smoothedAccel, newAccel);
      }
      V3<R> newVelocity = (forward * speed) + (smoothedAccel * dt);
      newVelocity = truncateLength(newVelocity, maxSpeed);
      speed = length(newVelocity);
      position = position + (newVelocity * dt);
      if (p.use2DProjection) newVelocity.y = 0;
      forward = normalize(newVelocity);
      if (p.use2DProjection) position.y = R(0.5f);
      R Lr = R(F.L);
      R pc[3] = {position.x, position.y, position.z};
      for (int a = 0; a < 3; ++a) {
        R x = pc[a];
        if (x >= Lr) x = x - Lr;
        else if (x < 0) { x = x + Lr; if (x >= Lr) x = 0; }
        pc[a] = x;
      }
      po[0] = pc[0]; po[1] = pc[1]; po[2] = pc[2]; po[3] = 1;
      ao[0] = smoothedAccel.x; ao[1] = smoothedAccel.y; ao[2] = smoothedAccel.z; ao[3] = A[3];
      wo[0] = forward.x; wo[1] = forward.y; wo[2] = forward.z; wo[3] = speed;
    }
  });
}

// splitmix64 (Steele, Lea, Flood 2014): the counter-based generator that
// replaces the Schooling plugin's time-seeded Mersenne Twister.
inline uint64_t splitmix64(uint64_t x) {
  uint64_t z = x + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
// Three uniforms in [0, 1) with 24 bits each, keyed on (seed, step, agent id).
inline void schoolRandom(uint32_t seed, uint32_t step, uint32_t id, float r[3]) {
  const uint64_t base = splitmix64(((uint64_t)seed << 32) | step);
  const uint64_t u1 = splitmix64(base ^ (uint64_t)id);
  const uint64_t u2 = splitmix64(u1);
  const float k = 5.9604644775390625e-08f;
  r[0] = (float)(uint32_t)(u1 >> 40) * k;
  r[1] = (float)(uint32_t)((u1 >> 16) & 0xFFFFFFu) * k;
  r[2] = (float)(uint32_t)(u2 >> 40) * k;
}

// The Schooling plugin's law per sorted slot (PlugIns/Schooling):
//   mode 1  Schooling_animateSchool (Schooling_kernel.cu:226-318)
//   mode 2  Schooling_repulsion (:64-95) -> Schooling_attractionOrientation
//           (:100-145, zone test inAttractionOrientationZone,
//           Schooling_resources.cu:34-71) -> Schooling_move (:150-221)
// The boundary term is the identity in the periodic world; positions wrap.
template <class R>
void schoolIntegrate(const Shared& S, const State<R>& st, State<R>& out, R* steerOut, uint32_t step, int threads) {
  const uint32_t stride = S.Mmax + 1;
  parallelFor(S.N, threads, [&](uint32_t b, uint32_t e) {
    std::vector<V3<R>> img(BRT_MAX_NEIGHBORS);
    for (uint32_t i = b; i < e; ++i) {
      const uint32_t id = S.sortedIds[i];
      const Flock& F = S.fl[S.flockOfAgent[id]];
      const brt_schooling_params& sc = F.p.schooling;
      const uint32_t* lst = &S.lists[(size_t)i * stride];
      const uint32_t n = lst[0];
      const R* P = &st.pos[4 * (size_t)i];
      const R* W = &st.fwd[4 * (size_t)i];
      const V3<R> myPos = v3(P), myFwd = v3(W);
      const float* pif = &S.sposf[4 * (size_t)i];
      for (uint32_t k = 0; k < n; ++k) {
        const uint32_t j = lst[1 + k];
        img[k] = imagePos<R>(F, &st.pos[4 * (size_t)j], pif, &S.sposf[4 * (size_t)j]);
      }
      V3<R> rep = mk<R>(0, 0, 0);
      uint32_t found = 0;
      for (uint32_t k = 0; k < n; ++k) {
        const V3<R> off = img[k] - myPos;
        const R dist = length(off);
        if (dist < R(sc.r_r)) { rep = rep + off / length(off); ++found; }
      }
      auto attractOrient = [&](bool blind) {
        V3<R> orient = myFwd / length(myFwd);
        V3<R> attr = mk<R>(0, 0, 0);
        for (uint32_t k = 0; k < n; ++k) {
          const V3<R> off = img[k] - myPos;
          const R dist = length(off);
          const bool in = blind ? (!(dist > R(sc.r_p)) && dot(myFwd, normalize(off)) > R(sc.eta)) : (dist < R(sc.r_p));
          if (in) {
            attr = attr + off / length(off);
            const V3<R> wj = v3(&st.fwd[4 * (size_t)lst[1 + k]]);
            orient = orient + wj / length(wj);
          }
        }
        return (attr * R(sc.w_a)) + (orient * R(sc.w_o));
      };
      V3<R> fwd, pos;
      if (sc.mode == 1) {
        V3<R> nf = mk<R>(-rep.x, -rep.y, -rep.z);
        if (found == 0) nf = attractOrient(false);
        if (F.p.use2DProjection) nf.y = 0;
        if (length(nf) > R(0)) nf = normalize(nf);
        fwd = vecLimitDeviationAngleUtility(nf, R(sc.theta), myFwd);
        pos = myPos + ((fwd * R(sc.s)) * R(0.1f));
      } else {
        V3<R> steer = rep;
        if (length(rep) > R(0)) {
          const V3<R> u = normalize(rep);
          steer = mk<R>(-u.x, -u.y, -u.z);
        }
        if (!(length(steer) > R(0))) {
          V3<R> nf = attractOrient(true);
          if (length(nf) > R(0)) nf = normalize(nf);
          steer = nf;
        }
        if (steerOut) {
          R* so = steerOut + 4 * (size_t)i;
          so[0] = steer.x; so[1] = steer.y; so[2] = steer.z; so[3] = 0;
        }
        V3<R> nf = steer;
        if (sc.randomDeviationWeight > 0.0f) {
          float r[3];
          schoolRandom(sc.seed, step, id, r);
          const R w = R(sc.randomDeviationWeight);
          const V3<R> rd = ((mk<R>(R(r[0]), R(r[1]), R(r[2])) * w) * R(2)) - (mk<R>(1, 1, 1) * w);
          nf = normalize(nf + rd);
        }
        fwd = vecLimitDeviationAngleUtility(nf, R(sc.theta), myFwd);
        pos = myPos + ((fwd * R(sc.s)) * R(0.2f));
      }
      if (F.p.use2DProjection) pos.y = R(0.5f);
      const R Lr = R(F.L);
      R pc[3] = {pos.x, pos.y, pos.z};
      for (int a = 0; a < 3; ++a) {
        R x = pc[a];
        if (x >= Lr) x = x - Lr;
        else if (x < 0) { x = x + Lr; if (x >= Lr) x = 0; }
        pc[a] = x;
      }
      R* po = &out.pos[4 * (size_t)i];
      R* wo = &out.fwd[4 * (size_t)i];
      po[0] = pc[0]; po[1] = pc[1]; po[2] = pc[2]; po[3] = 1;
      wo[0] = fwd.x; wo[1] = fwd.y; wo[2] = fwd.z; wo[3] = R(sc.s);
    }
  });
}

}  // namespace

extern "C" {
// Arguments of one oracle step.  Inputs are in agent-id order and use the
// working precision (float for mode 0, double for mode 1); so do the outputs.
typedef struct oracle_io {
  const void* pos4; const void* fwd4; const void* acc4; const void* feat; const void* stats4;
  void* pos4_out; void* fwd4_out; void* acc4_out; void* feat_out; void* stats4_out;
  uint32_t* sorted_keys; uint32_t* sorted_ids;     // N each
  uint32_t* cell_start; uint32_t* cell_end;        // total cells each
  uint32_t* lists;                                 // N * (Mmax+1), per sorted slot
  void* steer4;                                    // N * 4, per sorted slot
  uint32_t* scanned;                               // N, candidates examined per sorted slot
  uint32_t random_step;                            // Schooling random-stream step of this step
  uint32_t avoid_neighbors;                        // 1: crowd order, steerAndSlowToAvoidNeighbors for separation
  uint32_t move_away;                              // 1: the move-away-from-base stage after cohesion
  float avoid_base[3];                             // its base point
  float avoid_base_params[3];                      // (steering weight, acceleration factor, radius)
} oracle_io;
}  // extern "C"

namespace {
template <class R>
int stepImpl(uint32_t nflocks, const brt_params* params, R dt, const oracle_io* io, int threads) {
  Shared S;
  int rc = setupFlocks(S, nflocks, params);
  if (rc) return rc;
  const uint32_t N = S.N, Fd = S.Fmax;
  const R* pos = (const R*)io->pos4;
  const R* fwd = (const R*)io->fwd4;
  const R* acc = (const R*)io->acc4;
  const R* feat = (const R*)io->feat;
  const R* stats = (const R*)io->stats4;
  if (!pos || !fwd || !acc) return BRT_ERR_ARG;
  if (Fd && !feat) return BRT_ERR_ARG;
  std::vector<float> posf(4 * (size_t)N);
  for (size_t k = 0; k < 4 * (size_t)N; ++k) posf[k] = (float)pos[k];
  hashSortRanges(S, posf.data());
  neighborLists(S, threads);

  State<R> st, out;
  st.pos.resize(4 * (size_t)N); st.fwd.resize(4 * (size_t)N); st.acc.resize(4 * (size_t)N);
  st.stats.assign(4 * (size_t)N, R(0)); st.feat.resize((size_t)N * Fd);
  for (uint32_t s = 0; s < N; ++s) {
    size_t id = S.sortedIds[s];
    for (int a = 0; a < 4; ++a) {
      st.pos[4 * (size_t)s + a] = pos[4 * id + a];
      st.fwd[4 * (size_t)s + a] = fwd[4 * id + a];
      st.acc[4 * (size_t)s + a] = acc[4 * id + a];
      if (stats) st.stats[4 * (size_t)s + a] = stats[4 * id + a];
    }
    for (uint32_t a = 0; a < Fd; ++a) st.feat[(size_t)s * Fd + a] = feat[id * Fd + a];
  }
  out = st;
  std::vector<R> steer;
  if (io->steer4) steer.resize(4 * (size_t)N);
  if (params[0].schooling.mode != 0)
    schoolIntegrate<R>(S, st, out, io->steer4 ? steer.data() : nullptr, io->random_step, threads);
  else {
    const float moveAway[6] = {io->avoid_base[0], io->avoid_base[1], io->avoid_base[2],
                               io->avoid_base_params[0], io->avoid_base_params[1], io->avoid_base_params[2]};
    steerIntegrate<R>(S, st, dt, out, io->steer4 ? steer.data() : nullptr, io->avoid_neighbors != 0,
                      io->move_away ? moveAway : nullptr, threads);
  }

  // scatter back to agent-id order (OpenSteerWrapper_kernel.cu:324-331)
  R* po = (R*)io->pos4_out; R* wo = (R*)io->fwd4_out; R* ao = (R*)io->acc4_out;
  R* fo = (R*)io->feat_out; R* so = (R*)io->stats4_out;
  for (uint32_t s = 0; s < N; ++s) {
    size_t id = S.sortedIds[s];
    for (int a = 0; a < 4; ++a) {
      if (po) po[4 * id + a] = out.pos[4 * (size_t)s + a];
      if (wo) wo[4 * id + a] = out.fwd[4 * (size_t)s + a];
      if (ao) ao[4 * id + a] = out.acc[4 * (size_t)s + a];
      if (so) so[4 * id + a] = out.stats[4 * (size_t)s + a];
    }
    if (fo) for (uint32_t a = 0; a < Fd; ++a) fo[id * Fd + a] = out.feat[(size_t)s * Fd + a];
  }
  if (io->sorted_keys) std::memcpy(io->sorted_keys, S.sortedKeys.data(), 4 * (size_t)N);
  if (io->sorted_ids) std::memcpy(io->sorted_ids, S.sortedIds.data(), 4 * (size_t)N);
  if (io->cell_start) std::memcpy(io->cell_start, S.cellStart.data(), 4 * (size_t)S.Ctot);
  if (io->cell_end) std::memcpy(io->cell_end, S.cellEnd.data(), 4 * (size_t)S.Ctot);
  if (io->lists) std::memcpy(io->lists, S.lists.data(), 4 * S.lists.size());
  if (io->steer4) std::memcpy(io->steer4, steer.data(), sizeof(R) * steer.size());
  if (io->scanned) std::memcpy(io->scanned, S.scanned.data(), 4 * (size_t)N);
  return BRT_OK;
}
}  // namespace

extern "C" {

int oracle_step(int mode, uint32_t nflocks, const brt_params* params, float dt, const oracle_io* io, int threads) {
  if (!params || !io || nflocks == 0) return BRT_ERR_ARG;
  if (mode == 0) return stepImpl<float>(nflocks, params, dt, io, threads);
  if (mode == 1) return stepImpl<double>(nflocks, params, (double)dt, io, threads);
  return BRT_ERR_ARG;
}

int oracle_num_cells(uint32_t nflocks, const brt_params* params, uint32_t* cells) {
  Shared S;
  int rc = setupFlocks(S, nflocks, params);
  if (rc) return rc;
  *cells = S.Ctot;
  return BRT_OK;
}

int oracle_hardware_threads(void) { return (int)std::max(1u, std::thread::hardware_concurrency()); }

// The parameter defaults of the workloads, restated for the CPU side so that
// a CPU-only run never loads the CUDA library: the flocking demo's values
// (OpenSteerWrapperPlugIn install defaults, weights 1.5 / 1 / 1 of
// BehaveRT_Flocking.cpp), the unspecified constants fixed for this path
// (commonMass 1, sensing min radius 0, cosMaxAngle -2, maxBodiesPerCell
// unbounded, clustering steering off) and the Schooling install constants
// (SchoolingPlugIn.h:115-160).  A CPU test checks that the bytes equal the
// library's brt_params_default.
int oracle_params_default(brt_params* p) {
  if (!p) return BRT_ERR_ARG;
  std::memset(p, 0, sizeof(*p));
  p->numBodies = 4096;
  p->commonRadius = 1.0f;
  p->worldSize = 64.0f;
  p->cellSize = 4.0f;
  p->maxNeighbors = 16;
  p->commonSearchRadius = 4.0f;
  p->commonMaxSpeed = 1.0f;
  p->commonMaxForce = 0.1f;
  p->commonMass = 1.0f;
  const float w[3] = {1.5f, 1.0f, 1.0f};
  float* tri[3] = {p->separationParams, p->alignmentParams, p->cohesionParams};
  for (int k = 0; k < 3; ++k) { tri[k][0] = w[k]; tri[k][1] = 4.0f; tri[k][2] = -2.0f; }
  p->similarityStatsParams[0] = 0.01f;
  p->similarityStatsParams[1] = 0.1f;
  p->similarityStatsParams[2] = 0.001f;
  p->avgSimilarityController = 1.0f;
  p->schooling.theta = (float)std::cos(0.1);
  p->schooling.delta = 0.01f;
  p->schooling.r_r = 1.0f;
  p->schooling.r_p = 4.0f;
  p->schooling.eta = (float)std::cos(3.05);
  p->schooling.w_a = 1.0f;
  p->schooling.w_o = 16.0f;
  p->schooling.s = 3.0f;
  p->schooling.randomDeviationWeight = 0.1f;
  return BRT_OK;
}

}  // extern "C"
