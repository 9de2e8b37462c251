// brt_oracle_adjoint.cpp -- FP64 frozen-neighbour, frozen-branch forward and
// reverse-mode reference of the flocking step.  TEST INFRASTRUCTURE ONLY:
// used by tests/ and by the bench's CPU/accuracy leg as the checker of the
// CUDA adjoint, never by the library.
//
// Model.  One step maps every agent's (position p, unit forward f, speed s,
// smoothed acceleration a) to the next, with the neighbour list of every
// agent and step given (frozen) and every branch decision given (frozen):
// the inBoidNeighborhood result per neighbour and behaviour, the
// adjustRawSteeringForce low-speed and deviation-limit branches, and the two
// truncateLength clips.  With lists and branches fixed the step is a smooth
// function of the state and of the per-flock steering weights, so central
// finite differences and the hand-written reverse below agree to rounding.
// The forward restates the reference's operation sequence:
//   inBoidNeighborhood                OpenSteerWrapper_resources.cu:67-92
//   calcSeparation/Alignment/Cohesion OpenSteerWrapper_resources.cu:166-290
//   adjustRawSteeringForce            Core/common_resources.cu:234-254
//   vecLimitDeviationAngleUtility     Core/common_resources.cu:186-228
//   truncateLength                    Core/common_resources.cu:260-271
//   applySteeringForceSingle          OpenSteerWrapper_resources.cu:326-379
// plus the static sphere obstacle term of brt_oracle.cpp (no reference
// counterpart).  Neighbour and obstacle offsets use the minimum image of the
// periodic cube, which equals the cell-wrap image for neighbours closer than
// one cell.  Not covered (the CUDA adjoint rejects them too): feature
// clustering steering, kNN lists, use2DProjection and frozen agents
// (negative speed).
//
// Flag words, 4 per agent and step, in agent-id order:
//   [0] bit0 low-speed adjust branch taken, bit1 deviation limited,
//       bit2 force clipped to maxForce, bit3 velocity clipped to maxSpeed
//   [1] separation membership mask over list positions (bit k = neighbour k)
//   [2] alignment mask   [3] cohesion mask        (maxNeighbors <= 32)
#include "../include/behavert_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

struct D3 { double x, y, z; };
inline D3 d3(double x, double y, double z) { return D3{x, y, z}; }
inline D3 operator+(D3 a, D3 b) { return d3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline D3 operator-(D3 a, D3 b) { return d3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline D3 operator*(D3 a, double s) { return d3(a.x * s, a.y * s, a.z * s); }
inline D3 operator/(D3 a, double s) { return d3(a.x / s, a.y / s, a.z / s); }
inline D3& operator+=(D3& a, D3 b) { a = a + b; return a; }
inline D3& operator-=(D3& a, D3 b) { a = a - b; return a; }
inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double len(D3 a) { return std::sqrt(dot(a, a)); }
inline D3 normalize(D3 v) { return v * (1.0 / std::sqrt(dot(v, v))); }
// Adjoint of y = normalize(x): xbar = (I - y y^T) ybar / |x|.
inline D3 normalizeBar(D3 x, D3 ybar) {
  const double l = len(x);
  const D3 y = x / l;
  return (ybar - y * dot(y, ybar)) / l;
}
// Adjoint of y = x * (m / |x|) (a truncateLength that clipped).
inline D3 clipBar(D3 x, double m, D3 ybar) {
  const double l = len(x);
  const D3 h = x / l;
  return (ybar - h * dot(h, ybar)) * (m / l);
}

constexpr uint32_t kLow = 1u, kLimited = 2u, kClipF = 4u, kClipV = 8u;

struct Agent { D3 p, f, a; double s; };

struct FlockG {
  brt_params p;
  double L;
  uint32_t agentBase, n;
  double w[3];
  std::vector<double> obs;  // 4 per obstacle
};

inline double minImage(double d, double L) {
  if (d > 0.5 * L) return d - L;
  if (d < -0.5 * L) return d + L;
  return d;
}
inline D3 minImage3(D3 o, double L) { return d3(minImage(o.x, L), minImage(o.y, L), minImage(o.z, L)); }

bool inBoid(double dist, double cosA, double minR, double maxR, double cosMax) {
  if (dist < minR) return true;
  if (dist > maxR) return false;
  return cosA > cosMax;
}

inline double smoothAlpha(double dt) {
  if (!(dt > 0)) return 0.0;
  return std::min(std::max(9.0 * dt, (double)0.15f), (double)0.4f);
}
inline double lowSpeedLimit(const brt_params& p) { return (double)0.2f * (double)p.commonMaxSpeed; }

// Intermediates of one agent's step.
struct Rec {
  uint32_t n, mS, mA, mC, br;
  uint32_t cnt[3];
  D3 off[BRT_MAX_NEIGHBORS];
  D3 xs[3];
  bool on[3];
  D3 steer, adjusted, v, vT;
};

void stepAgent(uint32_t i, const std::vector<Agent>& S, const uint32_t* list, const uint32_t* frozen, const FlockG& F,
               double dt, Agent& out, Rec& r) {
  const brt_params& p = F.p;
  const Agent& A = S[i];
  r.n = list[0];
  D3 sum[3] = {d3(0, 0, 0), d3(0, 0, 0), d3(0, 0, 0)};
  r.cnt[0] = r.cnt[1] = r.cnt[2] = 0;
  r.mS = r.mA = r.mC = 0;
  for (uint32_t k = 0; k < r.n; ++k) {
    const Agent& B = S[list[1 + k]];
    const D3 o = minImage3(B.p - A.p, F.L);
    r.off[k] = o;
    const double d2 = dot(o, o), dist = std::sqrt(d2);
    bool is, ia, ic;
    if (frozen) {
      is = (frozen[1] >> k) & 1u; ia = (frozen[2] >> k) & 1u; ic = (frozen[3] >> k) & 1u;
    } else {
      const double cosA = dot(A.f, o * (1.0 / dist));
      const double minR = p.commonSensingMinRadius;
      is = inBoid(dist, cosA, minR, p.separationParams[1], p.separationParams[2]);
      ia = inBoid(dist, cosA, minR, p.alignmentParams[1], p.alignmentParams[2]);
      ic = inBoid(dist, cosA, minR, p.cohesionParams[1], p.cohesionParams[2]);
    }
    if (is) { sum[0] += o / (-d2); ++r.cnt[0]; r.mS |= 1u << k; }
    if (ia) { sum[1] += B.f; ++r.cnt[1]; r.mA |= 1u << k; }
    if (ic) { sum[2] += A.p + o; ++r.cnt[2]; r.mC |= 1u << k; }
  }
  r.xs[0] = r.cnt[0] ? sum[0] / (double)r.cnt[0] : d3(0, 0, 0);
  r.xs[1] = r.cnt[1] ? sum[1] / (double)r.cnt[1] - A.f : d3(0, 0, 0);
  r.xs[2] = r.cnt[2] ? sum[2] / (double)r.cnt[2] - A.p : d3(0, 0, 0);
  D3 steer = d3(0, 0, 0);
  for (int b = 0; b < 3; ++b) {
    // Memberships do not depend on the weight; a zero weight only drops the
    // term from the force, as the reference's `if (weight != 0)` does.
    r.on[b] = r.cnt[b] > 0;
    if (r.on[b] && F.w[b] != 0) steer += normalize(r.xs[b]) * F.w[b];
  }
  if (p.numObstacles && p.obstacleAvoidanceWeight != 0) {
    D3 s = d3(0, 0, 0);
    for (uint32_t o = 0; o < p.numObstacles; ++o) {
      const double* c = &F.obs[4 * o];
      const D3 off = minImage3(A.p - d3(c[0], c[1], c[2]), F.L);
      const double d = len(off), reach = c[3] + p.commonSearchRadius;
      if (d < reach && d > 0) s += off * ((1.0 - d / reach) / d);
    }
    steer += s * (double)p.obstacleAvoidanceWeight;
  }
  r.steer = steer;
  const double maxS = p.commonMaxSpeed, maxF = p.commonMaxForce, mass = p.commonMass;
  const double s0 = lowSpeedLimit(p);
  uint32_t br = 0;
  if (frozen) {
    br = frozen[0];
  } else if (!(A.s > s0) && !(steer.x == 0 && steer.y == 0 && steer.z == 0)) {
    br |= kLow;
    const double cosine = 1.0 - 2.0 * std::pow(A.s / s0, 20.0);
    const double L = len(steer);
    if (L != 0 && dot(steer / L, A.f) < cosine) br |= kLimited;
  }
  if ((br & kLow) && (br & kLimited)) {
    const double cosine = 1.0 - 2.0 * std::pow(A.s / s0, 20.0);
    const double L = len(steer);
    const D3 u = normalize(steer - A.f * dot(steer, A.f));
    const double pd = std::sqrt(1.0 - cosine * cosine);
    r.adjusted = (A.f * cosine + u * pd) * L;
  } else {
    r.adjusted = steer;
  }
  if (!frozen && len(r.adjusted) > maxF) br |= kClipF;
  const D3 clipped = (br & kClipF) ? r.adjusted * (maxF / len(r.adjusted)) : r.adjusted;
  const D3 newAccel = clipped / mass;
  const double alpha = smoothAlpha(dt);
  const D3 aNew = A.a + (newAccel - A.a) * alpha;
  r.v = A.f * A.s + aNew * dt;
  if (!frozen && len(r.v) > maxS) br |= kClipV;
  r.vT = (br & kClipV) ? r.v * (maxS / len(r.v)) : r.v;
  r.br = br;
  const D3 pn = A.p + r.vT * dt;
  auto wrap = [&](double x) {
    if (x >= F.L) return x - F.L;
    if (x < 0) { x += F.L; if (x >= F.L) x = 0; }
    return x;
  };
  out.p = d3(wrap(pn.x), wrap(pn.y), wrap(pn.z));
  out.f = normalize(r.vT);
  out.s = len(r.vT);
  out.a = aNew;
}

// Adjoint of one agent's step.  gOut is the adjoint of its new state;
// contributions go into G (adjoint of the old states of all agents) and gw
// (this flock's three weights).
void stepAgentBar(uint32_t i, const std::vector<Agent>& S, const uint32_t* list, const FlockG& F, double dt,
                  const Rec& r, const Agent& gOut, std::vector<Agent>& G, double* gw) {
  const brt_params& p = F.p;
  const Agent& A = S[i];
  const double maxS = p.commonMaxSpeed, maxF = p.commonMaxForce, mass = p.commonMass;
  const double alpha = smoothAlpha(dt);
  // p' = p + vT dt (the wrap is a translation); s' = |vT|; f' = normalize(vT)
  G[i].p += gOut.p;
  const double lvT = len(r.vT);
  const D3 gvT = gOut.p * dt + r.vT * (gOut.s / lvT) + normalizeBar(r.vT, gOut.f);
  const D3 gv = (r.br & kClipV) ? clipBar(r.v, maxS, gvT) : gvT;
  // v = f s + aNew dt
  G[i].f += gv * A.s;
  G[i].s += dot(A.f, gv);
  const D3 gaNew = gOut.a + gv * dt;
  // aNew = a + (newAccel - a) alpha, newAccel = clipped / mass
  G[i].a += gaNew * (1.0 - alpha);
  const D3 gClipped = gaNew * (alpha / mass);
  const D3 gAdj = (r.br & kClipF) ? clipBar(r.adjusted, maxF, gClipped) : gClipped;
  D3 gSteer = gAdj;
  if ((r.br & kLow) && (r.br & kLimited)) {
    // out = (f c + u pd) L, L = |steer|, u = normalize(steer - f (steer.f)),
    // c = 1 - 2 (s/s0)^20, pd = sqrt(1 - c^2)
    const double s0 = lowSpeedLimit(p);
    const double range = A.s / s0;
    const double c = 1.0 - 2.0 * std::pow(range, 20.0);
    const D3 src = r.steer, f = A.f;
    const double L = len(src);
    const D3 perp = src - f * dot(src, f);
    const double lp = len(perp);
    const D3 u = perp / lp;
    const double pd = std::sqrt(1.0 - c * c);
    const D3 dirOut = f * c + u * pd;
    D3 gSrc = (src / L) * dot(gAdj, dirOut);
    const D3 g = gAdj * L;
    D3 gF = g * c;
    double gC = dot(g, f);
    const double gPd = dot(g, u);
    const D3 gPerp = (g * pd - u * dot(u, g * pd)) / lp;
    const double k = dot(src, f);
    gSrc += gPerp;
    gF -= gPerp * k;
    const double gk = -dot(f, gPerp);
    gSrc += f * gk;
    gF += src * gk;
    if (pd > 0) gC += gPd * (-c / pd);
    G[i].s += gC * (-40.0 * std::pow(range, 19.0) / s0);
    G[i].f += gF;
    gSteer = gSrc;
  }
  D3 gx[3];
  for (int b = 0; b < 3; ++b) {
    gx[b] = d3(0, 0, 0);
    if (!r.on[b]) continue;
    gw[b] += dot(gSteer, normalize(r.xs[b]));
    gx[b] = normalizeBar(r.xs[b], gSteer * F.w[b]);
  }
  if (p.numObstacles && p.obstacleAvoidanceWeight != 0) {
    const D3 g = gSteer * (double)p.obstacleAvoidanceWeight;
    for (uint32_t o = 0; o < p.numObstacles; ++o) {
      const double* c = &F.obs[4 * o];
      const D3 off = minImage3(A.p - d3(c[0], c[1], c[2]), F.L);
      const double d = len(off), reach = c[3] + p.commonSearchRadius;
      // off (1/d - 1/R): Jacobian (1/d - 1/R) I - off off^T / d^3
      if (d < reach && d > 0) G[i].p += g * (1.0 / d - 1.0 / reach) - off * (dot(off, g) / (d * d * d));
    }
  }
  if (r.on[0]) {  // xs0 = sum_k (-o_k / |o_k|^2) / cnt, o_k = p_j - p_i
    const D3 gS = gx[0] / (double)r.cnt[0];
    for (uint32_t k = 0; k < r.n; ++k) {
      if (!((r.mS >> k) & 1u)) continue;
      const D3 o = r.off[k];
      const double d2 = dot(o, o);
      const D3 go = (gS / d2 - o * (2.0 * dot(o, gS) / (d2 * d2))) * -1.0;
      G[list[1 + k]].p += go;
      G[i].p -= go;
    }
  }
  if (r.on[1]) {  // xs1 = sum_k f_j / cnt - f_i
    const D3 gS = gx[1] / (double)r.cnt[1];
    for (uint32_t k = 0; k < r.n; ++k)
      if ((r.mA >> k) & 1u) G[list[1 + k]].f += gS;
    G[i].f -= gx[1];
  }
  if (r.on[2]) {  // xs2 = sum_k (p_i + o_k) / cnt - p_i, p_i + o_k = image of p_j
    const D3 gS = gx[2] / (double)r.cnt[2];
    for (uint32_t k = 0; k < r.n; ++k)
      if ((r.mC >> k) & 1u) G[list[1 + k]].p += gS;
    G[i].p -= gx[2];
  }
}

struct Setup {
  std::vector<FlockG> fl;
  std::vector<uint32_t> flockOf;
  uint32_t N = 0, stride = 0;
};

Setup makeSetup(uint32_t nflocks, const brt_params* params, const double* weights) {
  Setup s;
  uint32_t base = 0, mmax = 0;
  for (uint32_t f = 0; f < nflocks; ++f) {
    FlockG g;
    g.p = params[f];
    g.L = params[f].worldSize;
    g.agentBase = base;
    g.n = params[f].numBodies;
    const float dflt[3] = {params[f].separationParams[0], params[f].alignmentParams[0], params[f].cohesionParams[0]};
    for (int b = 0; b < 3; ++b) g.w[b] = weights ? weights[3 * f + b] : (double)dflt[b];
    for (uint32_t o = 0; o < params[f].numObstacles; ++o)
      for (int k = 0; k < 4; ++k) g.obs.push_back(params[f].obstacles[o][k]);
    base += g.n;
    mmax = std::max(mmax, params[f].maxNeighbors);
    s.fl.push_back(g);
  }
  s.N = base;
  s.stride = mmax + 1;
  s.flockOf.resize(s.N);
  for (uint32_t f = 0; f < nflocks; ++f)
    for (uint32_t i = 0; i < s.fl[f].n; ++i) s.flockOf[s.fl[f].agentBase + i] = f;
  return s;
}

std::vector<Agent> load(uint32_t N, const double* pos4, const double* fwd4, const double* acc4) {
  std::vector<Agent> S(N);
  for (uint32_t i = 0; i < N; ++i) {
    S[i].p = d3(pos4[4 * i], pos4[4 * i + 1], pos4[4 * i + 2]);
    S[i].f = d3(fwd4[4 * i], fwd4[4 * i + 1], fwd4[4 * i + 2]);
    S[i].s = fwd4[4 * i + 3];
    S[i].a = d3(acc4[4 * i], acc4[4 * i + 1], acc4[4 * i + 2]);
  }
  return S;
}

void store(const std::vector<Agent>& S, double* pos4, double* fwd4, double* acc4, double w0) {
  for (size_t i = 0; i < S.size(); ++i) {
    const Agent& A = S[i];
    pos4[4 * i] = A.p.x; pos4[4 * i + 1] = A.p.y; pos4[4 * i + 2] = A.p.z; pos4[4 * i + 3] = w0;
    fwd4[4 * i] = A.f.x; fwd4[4 * i + 1] = A.f.y; fwd4[4 * i + 2] = A.f.z; fwd4[4 * i + 3] = A.s;
    acc4[4 * i] = A.a.x; acc4[4 * i + 1] = A.a.y; acc4[4 * i + 2] = A.a.z; acc4[4 * i + 3] = 0;
  }
}

template <class Fn> void parFor(uint32_t n, int threads, Fn fn) {
  if (threads <= 1 || n < 2048) { fn(0u, n); return; }
  std::vector<std::thread> th;
  const uint32_t chunk = (n + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    const uint32_t b = t * chunk, e = std::min(n, b + chunk);
    if (b < e) th.emplace_back(fn, b, e);
  }
  for (auto& x : th) x.join();
}

void forwardSteps(const Setup& su, uint32_t T, double dt, const uint32_t* lists, const uint32_t* flags, uint32_t* flagsOut,
                  std::vector<std::vector<Agent>>* traj, std::vector<Agent>& S, int threads) {
  std::vector<Agent> Nx(su.N);
  for (uint32_t t = 0; t < T; ++t) {
    if (traj) (*traj)[t] = S;
    const uint32_t* L = lists + (size_t)t * su.N * su.stride;
    parFor(su.N, threads, [&](uint32_t b, uint32_t e) {
      Rec r;
      for (uint32_t i = b; i < e; ++i) {
        const uint32_t* fz = flags ? flags + ((size_t)t * su.N + i) * 4 : nullptr;
        stepAgent(i, S, L + (size_t)i * su.stride, fz, su.fl[su.flockOf[i]], dt, Nx[i], r);
        if (flagsOut) {
          uint32_t* w = flagsOut + ((size_t)t * su.N + i) * 4;
          w[0] = r.br; w[1] = r.mS; w[2] = r.mA; w[3] = r.mC;
        }
      }
    });
    std::swap(S, Nx);
  }
}

}  // namespace

extern "C" {

// FP64 trajectory of T steps with frozen neighbour lists and, when `flags`
// is given, frozen branch decisions (layout above).  lists: T * N * stride
// words by agent id, each row the count then the neighbours' agent ids in
// list order (stride = max maxNeighbors + 1).  weights: nflocks * 3
// (separation, alignment, cohesion) or NULL for the params'.  flags_out
// (optional) receives the decisions taken.  Final state in agent-id order.
int oracle_frozen_forward(uint32_t nflocks, const brt_params* params, const double* weights, uint32_t T, double dt,
                          const double* pos4, const double* fwd4, const double* acc4, const uint32_t* lists,
                          const uint32_t* flags, uint32_t* flags_out, double* pos4_out, double* fwd4_out,
                          double* acc4_out, int threads) {
  for (uint32_t f = 0; f < nflocks; ++f)
    if (params[f].maxNeighbors > 32) return BRT_ERR_CONFIG;
  Setup su = makeSetup(nflocks, params, weights);
  std::vector<Agent> S = load(su.N, pos4, fwd4, acc4);
  forwardSteps(su, T, dt, lists, flags, flags_out, nullptr, S, threads);
  store(S, pos4_out, fwd4_out, acc4_out, 1.0);
  return BRT_OK;
}

}  // extern "C"

namespace {

// The reverse sweep over a given trajectory (traj[t] = input state of step t).
void reverseSweep(const Setup& su, uint32_t nflocks, uint32_t T, double dt, const uint32_t* lists,
                  const uint32_t* flags, const std::vector<std::vector<Agent>>& traj, const double* gpos4_T,
                  const double* gfwd4_T, const double* gacc4_T, double* gpos4_0, double* gfwd4_0, double* gacc4_0,
                  double* gw) {
  std::vector<Agent> G = load(su.N, gpos4_T, gfwd4_T, gacc4_T);
  std::vector<double> gwAcc(3 * (size_t)nflocks, 0.0);
  const Agent zero{d3(0, 0, 0), d3(0, 0, 0), d3(0, 0, 0), 0.0};
  for (int t = (int)T - 1; t >= 0; --t) {
    std::vector<Agent> Gp(su.N, zero);
    const uint32_t* L = lists + (size_t)t * su.N * su.stride;
    Agent next;
    Rec r;
    for (uint32_t i = 0; i < su.N; ++i) {
      const uint32_t f = su.flockOf[i];
      const uint32_t* fz = flags ? flags + ((size_t)t * su.N + i) * 4 : nullptr;
      stepAgent(i, traj[t], L + (size_t)i * su.stride, fz, su.fl[f], dt, next, r);
      stepAgentBar(i, traj[t], L + (size_t)i * su.stride, su.fl[f], dt, r, G[i], Gp, &gwAcc[3 * f]);
    }
    G.swap(Gp);
  }
  store(G, gpos4_0, gfwd4_0, gacc4_0, 0.0);
  std::memcpy(gw, gwAcc.data(), sizeof(double) * gwAcc.size());
}

}  // namespace

extern "C" {

// Reverse mode of oracle_frozen_forward.  g*_T: adjoint of the final state
// (agent-id order; xyz of position / forward / acceleration, forward.w the
// adjoint of the speed).  Writes the adjoint of the initial state (same
// layout) and of the weights (nflocks * 3).
int oracle_frozen_reverse(uint32_t nflocks, const brt_params* params, const double* weights, uint32_t T, double dt,
                          const double* pos4, const double* fwd4, const double* acc4, const uint32_t* lists,
                          const uint32_t* flags, const double* gpos4_T, const double* gfwd4_T, const double* gacc4_T,
                          double* gpos4_0, double* gfwd4_0, double* gacc4_0, double* gw, int threads) {
  for (uint32_t f = 0; f < nflocks; ++f)
    if (params[f].maxNeighbors > 32) return BRT_ERR_CONFIG;
  Setup su = makeSetup(nflocks, params, weights);
  std::vector<std::vector<Agent>> traj(T);
  std::vector<Agent> S = load(su.N, pos4, fwd4, acc4);
  forwardSteps(su, T, dt, lists, flags, nullptr, &traj, S, threads);
  reverseSweep(su, nflocks, T, dt, lists, flags, traj, gpos4_T, gfwd4_T, gacc4_T, gpos4_0, gfwd4_0, gacc4_0, gw);
  return BRT_OK;
}

// The same reverse, linearised at a given trajectory instead of the FP64
// forward's: pos4_t / fwd4_t / acc4_t hold the input state of every step
// (T * N * 4 each, agent-id order), e.g. the FP32 states the GPU stepped
// through.  Against oracle_frozen_reverse this separates the effect of the
// trajectory (FP32 forward rounding) from the reverse arithmetic itself.
int oracle_frozen_reverse_at(uint32_t nflocks, const brt_params* params, const double* weights, uint32_t T, double dt,
                             const double* pos4_t, const double* fwd4_t, const double* acc4_t, const uint32_t* lists,
                             const uint32_t* flags, const double* gpos4_T, const double* gfwd4_T,
                             const double* gacc4_T, double* gpos4_0, double* gfwd4_0, double* gacc4_0, double* gw) {
  for (uint32_t f = 0; f < nflocks; ++f)
    if (params[f].maxNeighbors > 32) return BRT_ERR_CONFIG;
  Setup su = makeSetup(nflocks, params, weights);
  std::vector<std::vector<Agent>> traj(T);
  for (uint32_t t = 0; t < T; ++t) {
    const size_t o = (size_t)t * su.N * 4;
    traj[t] = load(su.N, pos4_t + o, fwd4_t + o, acc4_t + o);
  }
  reverseSweep(su, nflocks, T, dt, lists, flags, traj, gpos4_T, gfwd4_T, gacc4_T, gpos4_0, gfwd4_0, gacc4_0, gw);
  return BRT_OK;
}

}  // extern "C"
