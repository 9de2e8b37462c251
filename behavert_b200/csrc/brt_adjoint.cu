// brt_adjoint.cu -- reverse-mode kernels of the flocking step (no reference
// counterpart: BehaveRT has no differentiation).
//
// Model.  Neighbour sets and branch decisions are frozen per step: the
// reverse of a step recomputes, from the taped sorted state and neighbour
// list of that step, exactly the FP32 operation sequence of the forward
// (flockingSteer, obstacleSteer, integrate in brt_agent.cuh, so every branch
// decision agrees bit for bit with the forward that ran), then propagates the
// adjoint of the step's output back to its input and to the per-flock
// steering weights.  Per-agent adjoint arithmetic is FP32; the loss and the
// cross-agent weight-gradient reductions are FP64.
//
// Indexing.  A step reads its input in the canonical order left by the
// previous step, sorts it, and writes its output in its own sorted order.
// The adjoint of a step's output is therefore indexed by the step's sorted
// slot, and the adjoint of its input by canonical slot = the reorder's
// source slot `prev` of each sorted slot.
//
// Determinism.  The reverse of a step runs in two kernels, and no float is
// ever accumulated with an atomic:
//   emit    one thread per agent i: recomputes the forward, forms its own
//           adjoint terms and, for each list entry (i, k), the adjoint it
//           sends to the listed agent j, stored at the entry; the entry code
//           goes into j's in-list (an inbox whose positions come from an
//           atomic counter: the transposed neighbour list of the frozen step);
//   gather  one thread per agent j: adds the stored contributions of its
//           in-list to its own terms with an exact, order-free sum (64-bit
//           fixed point at a scale set by the largest term) and stores its
//           input adjoint (every canonical slot is written once).
// The weight adjoint is summed per agent over the steps in FP64 (each agent
// by its own thread, in step order) and reduced per flock in a fixed tree at
// the end.  Two runs from the same state give the same bits.
#include "brt_agent.cuh"
#include "brt_kernels.cuh"

namespace brt {

namespace {

// Adjoint of y = normalize(x): (I - y y^T) ybar / |x|.
__device__ __forceinline__ f3 normalizeBar(f3 x, f3 ybar) {
  const float l = len3(x);
  const f3 y = div3(x, l);
  return div3(sub3(ybar, mul3(y, dot3(y, ybar))), l);
}
// Adjoint of y = x * (m / |x|) (a truncateLength that clipped).
__device__ __forceinline__ f3 clipBar(f3 x, float m, f3 ybar) {
  const float l = len3(x);
  const f3 h = div3(x, l);
  return mul3(sub3(ybar, mul3(h, dot3(h, ybar))), m / l);
}

// Adjoint, with respect to the neighbour's offset o (|o|^2 = d2), of the
// separation term -o / |o|^2 given the adjoint g of the agent's separation
// sum divided by its count: -(g / d2 - 2 o (o . g) / d2^2).  Emit and gather
// evaluate it with this one sequence, so both sides hold the same bits.
__device__ __forceinline__ f3 separationBar(f3 o, float d2, f3 g) {
  return mul3(sub3(div3(g, d2), mul3(o, 2.0f * dot3(o, g) / (d2 * d2))), -1.0f);
}

// Compensated sum of float3 terms (Knuth's TwoSum per component; exact
// error terms, since the library is built without contraction).
struct Comp3 {
  f3 s = {0.f, 0.f, 0.f}, e = {0.f, 0.f, 0.f};
  __device__ __forceinline__ static void twoSum(float& sum, float& err, float t) {
    const float n = sum + t;
    const float bb = n - sum;
    err += (sum - (n - bb)) + (t - bb);
    sum = n;
  }
  __device__ __forceinline__ void add(f3 t) { twoSum(s.x, e.x, t.x); twoSum(s.y, e.y, t.y); twoSum(s.z, e.z, t.z); }
  __device__ __forceinline__ f3 value() const { return add3(s, e); }
};

// vecLimitDeviationAngle's result once the source is outside the cone
// (Core/common_resources.cu:214-227): the vector of the source's length on
// the cone's surface, in the plane of the source and the basis.
__device__ __forceinline__ f3 limitedDeviation(f3 source, float cosineOfConeAngle, f3 basis) {
  const float sourceLength = len3(source);
  const f3 perp = sub3(source, mul3(basis, dot3(source, basis)));
  const f3 unitPerp = normalize3(perp);
  const float perpDist = sqrtf(1.0f - (cosineOfConeAngle * cosineOfConeAngle));
  return mul3(add3(mul3(basis, cosineOfConeAngle), mul3(unitPerp, perpDist)), sourceLength);
}


}  // namespace

// Resident blocks per SM the two reverse kernels are compiled for: 6 caps them
// at 80 registers a thread (a few spills) and 24 resident warps; the
// uncapped builds (about 105 registers, 16 warps) were latency-bound and
// measured 5% slower on config 4's backward, 1.5% on config 3's.
constexpr int kAdjointMinBlocks = 6;

// Branch bits of the exported flag word (the oracle's frozen-branch layout).
constexpr uint32_t kBrLow = 1u, kBrLimited = 2u, kBrClipF = 4u, kBrClipV = 8u;

__global__ void __launch_bounds__(kAdjointThreads, kAdjointMinBlocks) adjointStepKernel(AdjointStepArgs A) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < A.n;
  uint32_t f = 0;
  float gw[3] = {0.0f, 0.0f, 0.0f};
  if (valid) {
    f = A.nflocks == 1 ? 0u : flockOfSlot(A.agentBase, A.nflocks, i);
    const FlockDev& fl = A.flocks[f];
    const float4 p4 = __ldg(&A.posS[i]);
    const float4 w4 = __ldg(&A.fwdS[i]);
    const float4 a4 = __ldg(&A.accS[i]);
    const AgentCtx a = makeCtx(p4, w4, fl);
    const uint32_t* lst = A.lists + (size_t)i * A.listStride;
    const uint32_t n = lst[0];
    const uint32_t self = __ldg(&A.prev[i]);

    // The adjoint of this step's output.
    const float4 gOp = A.gOutP[i], gOf = A.gOutF[i], gOa = A.gOutA[i];

    // --- forward recomputation (flockingSteer's sequence) -----------------
    // Two evaluations of the three neighbour sums.  The forward's own order
    // (x, steer) decides every branch exactly as the forward did.  The
    // adjoint is linearised at the sums taken in offset form with
    // compensated (TwoSum) accumulation (xL, steerL): the cohesion sum in
    // the forward's form, (sum of positions) / n - own position, cancels
    // coordinates of the world's size down to about one and keeps only
    // ~1e-4 of its value, which the 50-step reverse would amplify.
    f3 sSep = mk3(0.f, 0.f, 0.f), sAli = mk3(0.f, 0.f, 0.f), sCoh = mk3(0.f, 0.f, 0.f);
    Comp3 cpSep, cpAli, cpCoh;
    uint32_t cSep = 0, cAli = 0, cCoh = 0, mS = 0, mA = 0, mC = 0;
    // Memberships as the flock kernel decides them: with the angle test
    // inactive (cosFree), exact squared-distance thresholds; otherwise the
    // distance and the cosine (both forms decide the same, bit for bit).
    const bool cosFree = dot3(a.fwd, a.fwd) * 1.002f < fl.cosBound2;
    for (uint32_t k = 0; k < n; ++k) {
      const uint32_t j = lst[1 + k];
      const f3 other = neighborImage(a, __ldg(&A.posS[j]), fl);
      const f3 offset = sub3(other, a.pos);
      const float d2 = dot3(offset, offset);
      bool inS, inA, inC;
      if (cosFree && d2 >= 1e-30f) {
        const bool lo = d2 < fl.minT;
        inS = lo || !(d2 > fl.sepT);
        inA = lo || !(d2 > fl.aliT);
        inC = lo || !(d2 > fl.cohT);
      } else {
        const float dist = sqrtf(d2);
        const f3 nrm = mul3(offset, 1.0f / dist);
        const float cosAngle = dot3(a.fwd, nrm);
        inS = inBoid(dist, cosAngle, fl.minR, fl.sep[1], fl.sep[2]);
        inA = inBoid(dist, cosAngle, fl.minR, fl.ali[1], fl.ali[2]);
        inC = inBoid(dist, cosAngle, fl.minR, fl.coh[1], fl.coh[2]);
      }
      if (inS) {
        const f3 t = div3(offset, -d2);
        sSep = add3(sSep, t);
        cpSep.add(t);
        ++cSep;
        mS |= 1u << k;
      }
      if (inA) {
        const f3 fj = xyz(__ldg(&A.fwdS[j]));
        sAli = add3(sAli, fj);
        cpAli.add(sub3(fj, a.fwd));
        ++cAli;
        mA |= 1u << k;
      }
      if (inC) {
        sCoh = add3(sCoh, other);
        cpCoh.add(offset);
        ++cCoh;
        mC |= 1u << k;
      }
    }
    const float w[3] = {fl.sep[0], fl.ali[0], fl.coh[0]};
    f3 x[3], xL[3], u[3], uL[3];
    const uint32_t cnt[3] = {cSep, cAli, cCoh};
    x[0] = cSep ? div3(sSep, (float)cSep) : sSep;
    x[1] = cAli ? sub3(div3(sAli, (float)cAli), a.fwd) : sAli;
    x[2] = cCoh ? sub3(div3(sCoh, (float)cCoh), a.pos) : sCoh;
    xL[0] = cSep ? div3(cpSep.value(), (float)cSep) : sSep;
    xL[1] = cAli ? div3(cpAli.value(), (float)cAli) : sAli;
    xL[2] = cCoh ? div3(cpCoh.value(), (float)cCoh) : sCoh;
    f3 steer = mk3(0.f, 0.f, 0.f), steerL = mk3(0.f, 0.f, 0.f);
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      u[b] = cnt[b] ? normalize3(x[b]) : x[b];
      uL[b] = cnt[b] ? normalize3(xL[b]) : xL[b];
      if (w[b] != 0.0f) {
        steer = add3(mul3(u[b], w[b]), steer);
        steerL = add3(mul3(uL[b], w[b]), steerL);
      }
    }
    if (fl.numObstacles && fl.obsW != 0.0f) {
      steer = obstacleSteer(a, fl, A.obstacles, A.obsMask, steer);
      steerL = obstacleSteer(a, fl, A.obstacles, A.obsMask, steerL);
    }

    f3 gSteer = mk3(0.f, 0.f, 0.f);
    f3 selfP = xyz(gOp), selfF = mk3(0.f, 0.f, 0.f), selfA = xyz(gOa);
    float selfS = 0.0f;
    uint32_t br = 0;
    if (a.speed < 0.0f) {
      // A frozen agent keeps position and acceleration; its forward output
      // is the steering force itself.
      gSteer = xyz(gOf);
    } else {
      // integrate()'s sequence
      const float maxS = fl.maxSpeed, maxF = fl.maxForce, mass = fl.mass, dt = A.dt;
      const float speed = a.speed;
      const f3 fwd = a.fwd;
      const float s0 = 0.2f * maxS;
      f3 adjusted = steer;
      float cosine = 0.0f;
      if (!(speed > s0) && !(steer.x == 0.0f && steer.y == 0.0f && steer.z == 0.0f)) {
        br |= kBrLow;
        const float range = speed / s0;
        cosine = 1.0f + ((-1.0f - 1.0f) * pow20f(range));
        const float srcLen = len3(steer);
        if (srcLen != 0.0f && !(dot3(div3(steer, srcLen), fwd) >= cosine)) br |= kBrLimited;
        adjusted = vecLimitDeviationAngle(steer, cosine, fwd);
      }
      if (!(len3(adjusted) <= maxF)) br |= kBrClipF;
      const f3 clipped = truncateLength(adjusted, maxF);
      const f3 newAccel = div3(clipped, mass);
      f3 smoothed = xyz(a4);
      float alpha = 0.0f;
      if (dt > 0.0f) {
        alpha = clampf(clampf(9.0f * dt, 0.15f, 0.4f), 0.0f, 1.0f);
        smoothed = add3(smoothed, mul3(sub3(newAccel, smoothed), alpha));
      }
      const f3 vF = add3(mul3(fwd, speed), mul3(smoothed, dt));
      if (!(len3(vF) <= maxS)) br |= kBrClipV;

      // The same integration from steerL, through the branches taken above:
      // the point the adjoint is linearised at.
      if ((br & kBrLow) && (br & kBrLimited)) adjusted = limitedDeviation(steerL, cosine, fwd);
      else adjusted = steerL;
      const f3 clippedL = (br & kBrClipF) ? mul3(adjusted, maxF / len3(adjusted)) : adjusted;
      f3 smoothedL = xyz(a4);
      if (dt > 0.0f) smoothedL = add3(smoothedL, mul3(sub3(div3(clippedL, mass), smoothedL), alpha));
      const f3 v = add3(mul3(fwd, speed), mul3(smoothedL, dt));
      const f3 vT = (br & kBrClipV) ? mul3(v, maxS / len3(v)) : v;
      steer = steerL;

      // --- adjoint of the integration --------------------------------------
      const float lvT = len3(vT);
      f3 gvT = add3(mul3(xyz(gOp), dt), mul3(vT, gOf.w / lvT));
      gvT = add3(gvT, normalizeBar(vT, xyz(gOf)));
      const f3 gv = (br & kBrClipV) ? clipBar(v, maxS, gvT) : gvT;
      selfF = mul3(gv, speed);
      selfS = dot3(fwd, gv);
      const f3 gaNew = add3(xyz(gOa), mul3(gv, dt));
      selfA = mul3(gaNew, 1.0f - alpha);
      const f3 gClipped = mul3(gaNew, alpha / mass);
      const f3 gAdj = (br & kBrClipF) ? clipBar(adjusted, maxF, gClipped) : gClipped;
      gSteer = gAdj;
      if ((br & kBrLow) && (br & kBrLimited)) {
        // adjusted = (fwd c + u pd) L with L = |steer|,
        // u = normalize(steer - fwd (steer . fwd)), pd = sqrt(1 - c^2),
        // c = 1 - 2 (speed / s0)^20.
        const float range = speed / s0;
        const float L = len3(steer);
        const float kk = dot3(steer, fwd);
        const f3 perp = sub3(steer, mul3(fwd, kk));
        const float lp = len3(perp);
        const f3 uu = div3(perp, lp);
        const float pd = sqrtf(1.0f - cosine * cosine);
        const f3 dirOut = add3(mul3(fwd, cosine), mul3(uu, pd));
        f3 gSrc = mul3(div3(steer, L), dot3(gAdj, dirOut));
        const f3 g = mul3(gAdj, L);
        f3 gF = mul3(g, cosine);
        float gC = dot3(g, fwd);
        const float gPd = dot3(g, uu);
        const f3 gu = mul3(g, pd);
        const f3 gPerp = div3(sub3(gu, mul3(uu, dot3(uu, gu))), lp);
        gSrc = add3(gSrc, gPerp);
        gF = sub3(gF, mul3(gPerp, kk));
        const float gk = -dot3(fwd, gPerp);
        gSrc = add3(gSrc, mul3(fwd, gk));
        gF = add3(gF, mul3(steer, gk));
        if (pd > 0.0f) gC += gPd * (-cosine / pd);
        selfS += gC * (-40.0f * pow19f(range) / s0);
        selfF = add3(selfF, gF);
        gSteer = gSrc;
      }
    }

    // --- adjoint of the steering force -------------------------------------
    f3 gx[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      gx[b] = mk3(0.f, 0.f, 0.f);
      if (!cnt[b]) continue;
      gw[b] = dot3(gSteer, uL[b]);
      gx[b] = normalizeBar(xL[b], mul3(gSteer, w[b]));
    }
    if (fl.numObstacles && fl.obsW != 0.0f) {
      const f3 g = mul3(gSteer, fl.obsW);
      const float L = fl.L, hL = 0.5f * fl.L;
      for (uint64_t bits = obstacleBits(a, fl, A.obsMask); bits; bits &= bits - 1ull) {
        const uint32_t o = (uint32_t)__ffsll((long long)bits) - 1u;
        const float4 c = __ldg(&A.obstacles[fl.obsBase + o]);
        f3 off = sub3(a.pos, xyz(c));
        if (off.x > hL) off.x = off.x - L; else if (off.x < -hL) off.x = off.x + L;
        if (off.y > hL) off.y = off.y - L; else if (off.y < -hL) off.y = off.y + L;
        if (off.z > hL) off.z = off.z - L; else if (off.z < -hL) off.z = off.z + L;
        const float d = len3(off);
        const float reach = c.w + fl.radius;
        if (d < reach && d > 0.0f) {
          // off (1/d - 1/reach): Jacobian (1/d - 1/reach) I - off off^T / d^3
          selfP = add3(selfP, sub3(mul3(g, 1.0f / d - 1.0f / reach), mul3(off, dot3(off, g) / (d * d * d))));
        }
      }
    }
    const f3 gSs = cSep ? div3(gx[0], (float)cSep) : gx[0];
    const f3 gSa = cAli ? div3(gx[1], (float)cAli) : gx[1];
    const f3 gSc = cCoh ? div3(gx[2], (float)cCoh) : gx[2];
    selfF = sub3(selfF, gx[1]);
    selfP = sub3(selfP, gx[2]);
    // Every list entry (i, k) with a contribution: the adjoint it sends to
    // the agent j it lists, stored at the entry, and the entry into j's
    // in-list.  The separation term's own share goes to selfP (in list order).
    // Entries go kEmitGroup at a time: the group's in-list positions are
    // reserved by atomics issued back to back, so their round trips overlap
    // (a store waiting on its own atomic would otherwise hold up the next
    // entry's atomic).  Positions only place terms the gather sums order-free.
    constexpr int kEmitGroup = 4;
    for (uint32_t m = mS | mA | mC; m;) {
      uint32_t kk[kEmitGroup], jj[kEmitGroup], q[kEmitGroup];
#pragma unroll
      for (int u = 0; u < kEmitGroup; ++u) {
        kk[u] = m ? (uint32_t)__ffs(m) - 1u : kNoEntry;
        m &= m - 1u;
        jj[u] = kk[u] != kNoEntry ? lst[1 + kk[u]] : 0u;
      }
#pragma unroll
      for (int u = 0; u < kEmitGroup; ++u) q[u] = kk[u] != kNoEntry ? atomicAdd(&A.inCount[jj[u]], 1u) : 0u;
#pragma unroll
      for (int u = 0; u < kEmitGroup; ++u) {
        if (kk[u] == kNoEntry) break;
        const uint32_t k = kk[u], j = jj[u];
        f3 gp = mk3(0.f, 0.f, 0.f);
        if ((mS >> k) & 1u) {
          const f3 other = neighborImage(a, __ldg(&A.posS[j]), fl);
          const f3 o = sub3(other, a.pos);
          const f3 go = separationBar(o, dot3(o, o), gSs);
          gp = add3(gp, go);
          selfP = sub3(selfP, go);
        }
        if ((mC >> k) & 1u) gp = add3(gp, gSc);
        const f3 gf = ((mA >> k) & 1u) ? gSa : mk3(0.f, 0.f, 0.f);
        const float4 c0 = make_float4(gp.x, gp.y, gp.z, gf.x), c1 = make_float4(gf.y, gf.z, 0.0f, 0.0f);
        if (q[u] < A.inCap) {
          float4* slot = A.inbox + 2 * ((size_t)j * A.inCap + q[u]);
          slot[0] = c0;
          slot[1] = c1;
        } else {
          const uint32_t e = i * A.entryStride + k;
          A.contrib[2 * (size_t)e + 0] = c0;
          A.contrib[2 * (size_t)e + 1] = c1;
          A.ovNext[e] = atomicExch(&A.ovHead[j], e);
        }
      }
    }
    A.selfP[i] = make_float4(selfP.x, selfP.y, selfP.z, 0.0f);
    A.selfF[i] = make_float4(selfF.x, selfF.y, selfF.z, selfS);
    if (self < A.n) A.gInA[self] = make_float4(selfA.x, selfA.y, selfA.z, 0.0f);

    const uint32_t id = __ldg(&A.idS[i]);
    double* acc = A.accW + 3 * (size_t)id;
    acc[0] += (double)gw[0];
    acc[1] += (double)gw[1];
    acc[2] += (double)gw[2];

    if (A.exportFlags) {
      reinterpret_cast<uint4*>(A.exportFlags)[id] = make_uint4(br, mS, mA, mC);
      uint32_t* row = A.exportLists + (size_t)id * A.listStride;
      row[0] = n;
      for (uint32_t k = 0; k < n; ++k) row[1 + k] = __ldg(&A.idS[lst[1 + k]]);
    }
    if (A.exportState) {
      A.exportState[3 * (size_t)id + 0] = p4;
      A.exportState[3 * (size_t)id + 1] = w4;
      A.exportState[3 * (size_t)id + 2] = a4;
    }
  }
}

// The gather's sums are exact and order-free.  Per component, every term
// (the agent's own and each in-list entry's) is scaled by 2^sh, sh fixed by
// the largest magnitude among them and the number of terms, rounded to an
// integer and added in 64-bit integers, which is exact and associative; the
// total is rounded to float once.  Terms below 2^-sh of the largest round to
// zero (their share of the float result is below its last bit).  So the
// result does not depend on the order the in-list was filled in, and no sort
// is needed.
struct ExactSum6 {
  float mx[6];
  int sh[6];
  float up[6], down[6];  // 2^sh and 2^-sh when both are normal floats, else 0 (ldexpf then)
  long long acc[6];
  bool finite = true;
  __device__ __forceinline__ void seeMax(const float* t) {
#pragma unroll
    for (int c = 0; c < 6; ++c) mx[c] = fmaxf(mx[c], fabsf(t[c]));
  }
  __device__ __forceinline__ void scales(uint32_t terms) {
    const int headroom = 32 - __clz((int)terms);  // bits to hold the count of terms
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      if (!isfinite(mx[c])) finite = false;
      // mx = f * 2^ex with f in [0.5, 1): the biased exponent of a normal
      // float minus 126, frexpf for the rest (zero and subnormals)
      const uint32_t bits = __float_as_uint(mx[c]);
      const int be = (int)((bits >> 23) & 0xFFu);
      int ex = be - 126;
      if (be == 0) {
        ex = 0;
        if (mx[c] > 0.0f) frexpf(mx[c], &ex);
      }
      sh[c] = 62 - headroom - ex;  // |term| * 2^sh < 2^(62 - headroom)
      const bool fast = sh[c] >= -126 && sh[c] <= 127;
      up[c] = fast ? __uint_as_float((uint32_t)(sh[c] + 127) << 23) : 0.0f;
      down[c] = fast ? __uint_as_float((uint32_t)(127 - sh[c]) << 23) : 0.0f;
      acc[c] = 0;
    }
  }
  // term * 2^sh, exact (a power-of-two scale that neither overflows nor,
  // for any term that rounds to a nonzero integer, underflows)
  __device__ __forceinline__ float scaled(float t, int c) const { return up[c] != 0.0f ? t * up[c] : ldexpf(t, sh[c]); }
  __device__ __forceinline__ void add(const float* t) {
#pragma unroll
    for (int c = 0; c < 6; ++c) acc[c] += __float2ll_rn(scaled(t[c], c));
  }
  __device__ __forceinline__ float value(int c) const {
    const float v = __ll2float_rn(acc[c]);
    return down[c] != 0.0f ? v * down[c] : ldexpf(v, -sh[c]);
  }
};

__device__ __forceinline__ void termsOf(const float4 c0, const float4 c1, float* t) {
  t[0] = c0.x; t[1] = c0.y; t[2] = c0.z; t[3] = c0.w; t[4] = c1.x; t[5] = c1.y;
}

// kGatherLanes consecutive lanes gather one agent: lane `sub` takes inbox
// entries sub, sub + kGatherLanes, ... (the group reads the agent's inbox
// block coalesced, once, and keeps its terms in registers for the second
// pass) and every kGatherLanes-th overflow entry.  The maxima and the
// integer sums combine across the lanes exactly (both are associative), so
// the split changes no bit.
constexpr uint32_t kGatherLanes = 8;
constexpr uint32_t kGatherPerLane = 8;  // inbox entries a lane holds: inCap <= 64

__global__ void __launch_bounds__(kAdjointThreads, kAdjointMinBlocks) adjointGatherKernel(AdjointStepArgs A) {
  const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t j = gt / kGatherLanes, sub = gt % kGatherLanes;
  const bool valid = j < A.n;
  uint32_t cnt = 0, head = kNoEntry, inBox = 0;
  float self[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  float selfS = 0.0f;
  if (valid) {
    cnt = A.inCount[j];
    inBox = min(cnt, A.inCap);
    if (cnt > A.inCap) head = A.ovHead[j];
    const float4 sp = A.selfP[j], sf = A.selfF[j];
    self[0] = sp.x; self[1] = sp.y; self[2] = sp.z; self[3] = sf.x; self[4] = sf.y; self[5] = sf.z;
    selfS = sf.w;
  }
  // this lane's inbox terms, in registers
  float tk[kGatherPerLane][6];
  const float4* box = A.inbox + 2 * (size_t)j * A.inCap;
  ExactSum6 S;
#pragma unroll
  for (int c = 0; c < 6; ++c) S.mx[c] = fabsf(self[c]);
#pragma unroll
  for (uint32_t r = 0; r < kGatherPerLane; ++r) {
    const uint32_t q = sub + r * kGatherLanes;
    if (q < inBox) {
      termsOf(box[2 * q], box[2 * q + 1], tk[r]);
      S.seeMax(tk[r]);
    }
  }
  float t[6];
  uint32_t r = 0;
  for (uint32_t e = head; e != kNoEntry; e = A.ovNext[e], ++r)
    if (r % kGatherLanes == sub) { termsOf(A.contrib[2 * (size_t)e], A.contrib[2 * (size_t)e + 1], t); S.seeMax(t); }
  // the group's maxima (the lanes of one agent are consecutive in the warp)
#pragma unroll
  for (int c = 0; c < 6; ++c)
#pragma unroll
    for (uint32_t o = 1; o < kGatherLanes; o <<= 1) S.mx[c] = fmaxf(S.mx[c], __shfl_xor_sync(0xFFFFFFFFu, S.mx[c], o));
  S.scales(cnt + 1u);
  const bool finite = S.finite;  // the same in every lane of the group (same maxima)
  if (finite) {
    if (sub == 0) S.add(self);
#pragma unroll
    for (uint32_t rr = 0; rr < kGatherPerLane; ++rr)
      if (sub + rr * kGatherLanes < inBox) S.add(tk[rr]);
    r = 0;
    for (uint32_t e = head; e != kNoEntry; e = A.ovNext[e], ++r)
      if (r % kGatherLanes == sub) { termsOf(A.contrib[2 * (size_t)e], A.contrib[2 * (size_t)e + 1], t); S.add(t); }
  }
#pragma unroll
  for (int c = 0; c < 6; ++c)
#pragma unroll
    for (uint32_t o = 1; o < kGatherLanes; o <<= 1) S.acc[c] += __shfl_xor_sync(0xFFFFFFFFu, S.acc[c], o);
  if (!valid || sub != 0) return;
  A.inCount[j] = 0u;  // clean for the next-earlier step
  if (cnt > A.inCap) A.ovHead[j] = kNoEntry;
  float res[6];
  if (finite) {
#pragma unroll
    for (int c = 0; c < 6; ++c) res[c] = S.value(c);
  } else {
    // a non-finite term: no exact sum; a plain one (not finite either)
#pragma unroll
    for (int c = 0; c < 6; ++c) res[c] = self[c];
    for (uint32_t q = 0; q < inBox; ++q) {
      termsOf(box[2 * q], box[2 * q + 1], t);
#pragma unroll
      for (int c = 0; c < 6; ++c) res[c] += t[c];
    }
    for (uint32_t e = head; e != kNoEntry; e = A.ovNext[e]) {
      termsOf(A.contrib[2 * (size_t)e], A.contrib[2 * (size_t)e + 1], t);
#pragma unroll
      for (int c = 0; c < 6; ++c) res[c] += t[c];
    }
  }
  const uint32_t tj = __ldg(&A.prev[j]);
  if (tj >= A.n) return;  // only a corrupted step leaves such a source slot
  A.gInP[tj] = make_float4(res[0], res[1], res[2], 0.0f);
  A.gInF[tj] = make_float4(res[3], res[4], res[5], selfS);
}

// Per-flock sums of `width` doubles per item over flock f's items
// [agentBase[f], agentBase[f+1]), in an order fixed by the sizes alone:
// block (f, b) sums part b of the flock (kReduceParts equal parts; each
// thread a fixed stride of items, then a fixed tree in shared memory), and
// flockReducePartsKernel adds the parts in order.
__global__ void __launch_bounds__(256) flockReduceKernel(FlockReduceArgs A) {
  __shared__ double sh[3][256];
  const uint32_t f = blockIdx.x, b = blockIdx.y;
  const uint32_t a0 = __ldg(&A.agentBase[f]), a1 = __ldg(&A.agentBase[f + 1]);
  const uint32_t part = (a1 - a0 + kReduceParts - 1) / kReduceParts;
  const uint32_t p0 = a0 + b * part, p1 = min(a1, p0 + part);
  const uint32_t w = A.width;
  double s[3] = {0.0, 0.0, 0.0};
  for (uint32_t id = p0 + threadIdx.x; id < p1; id += 256u)
    for (uint32_t c = 0; c < w; ++c) s[c] += A.vals[(size_t)w * id + c];
  for (int c = 0; c < 3; ++c) sh[c][threadIdx.x] = s[c];
  __syncthreads();
  for (uint32_t h = 128; h > 0; h >>= 1) {
    if (threadIdx.x < h)
      for (int c = 0; c < 3; ++c) sh[c][threadIdx.x] += sh[c][threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (uint32_t c = 0; c < w; ++c) A.partial[((size_t)f * kReduceParts + b) * w + c] = sh[c][0];
}

__global__ void __launch_bounds__(256) flockReducePartsKernel(FlockReduceArgs A) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= A.nflocks * A.width) return;
  const uint32_t f = t / A.width, c = t - f * A.width;
  double s = 0.0;
  for (uint32_t b = 0; b < kReduceParts; ++b) s += A.partial[((size_t)f * kReduceParts + b) * A.width + c];
  A.out[t] = s;
}

// Loss = sum over flocks of the mean squared minimum-image distance between
// final and target positions (FP64): each agent's term into lossTerm (by
// canonical slot; flocks own fixed slot ranges), reduced per flock in a fixed
// order by flockReduceKernel; and the unscaled terminal position adjoint
// 2 d / n_f (canonical order).
__global__ void __launch_bounds__(256) lossKernel(LossArgs A) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const uint32_t f = A.nflocks == 1 ? 0u : flockOfSlot(A.agentBase, A.nflocks, i);
  const FlockDev& fl = A.flocks[f];
  const float4 p = __ldg(&A.posA[i]);
  const float4 t = __ldg(&A.target[__ldg(&A.idA[i])]);
  const double L = fl.L, hL = 0.5 * (double)fl.L;
  double d[3] = {(double)p.x - (double)t.x, (double)p.y - (double)t.y, (double)p.z - (double)t.z};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (d[c] > hL) d[c] -= L; else if (d[c] < -hL) d[c] += L;
  }
  const double inv = 1.0 / (double)fl.n;
  A.lossTerm[i] = (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) * inv;
  A.gT[i] = make_float4((float)(2.0 * d[0] * inv), (float)(2.0 * d[1] * inv), (float)(2.0 * d[2] * inv), 0.0f);
}

// Terminal adjoint of the last step's output (its sorted order = the final
// canonical order): scale[f] * gT plus optional id-ordered extra adjoints.
__global__ void __launch_bounds__(256) adjointSeedKernel(SeedArgs A) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const uint32_t f = A.nflocks == 1 ? 0u : flockOfSlot(A.agentBase, A.nflocks, i);
  const float s = A.scale ? A.scale[f] : 1.0f;
  const float4 g = A.gT ? A.gT[i] : make_float4(0.f, 0.f, 0.f, 0.f);
  float4 p = make_float4(g.x * s, g.y * s, g.z * s, 0.0f);
  float4 fw = make_float4(0.f, 0.f, 0.f, 0.f), ac = make_float4(0.f, 0.f, 0.f, 0.f);
  const uint32_t id = __ldg(&A.idA[i]);
  if (A.extraP) { const float4 e = A.extraP[id]; p.x += e.x; p.y += e.y; p.z += e.z; }
  if (A.extraF) fw = A.extraF[id];
  if (A.extraA) ac = A.extraA[id];
  A.gP[i] = p;
  A.gF[i] = fw;
  A.gA[i] = ac;
}

// Adjoint of the initial state in agent-id order, plus the adjoint with
// respect to the initial velocity v = forward * speed:
//   dL/dv = (dL/ds) f + (I - f f^T) dL/df / s.
__global__ void __launch_bounds__(256) adjointOutKernel(OutArgs A) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const uint32_t id = __ldg(&A.id0[i]);
  const float4 gp = A.gP[i], gf = A.gF[i], ga = A.gA[i];
  if (A.outP) A.outP[id] = make_float4(gp.x, gp.y, gp.z, 0.0f);
  if (A.outF) A.outF[id] = gf;
  if (A.outA) A.outA[id] = make_float4(ga.x, ga.y, ga.z, 0.0f);
  if (A.outV) {
    const float4 w = __ldg(&A.fwd0[i]);
    const f3 f = xyz(w);
    const f3 g = xyz(gf);
    const f3 t = div3(sub3(g, mul3(f, dot3(f, g))), w.w);
    const f3 v = add3(mul3(f, gf.w), t);
    A.outV[id] = make_float4(v.x, v.y, v.z, 0.0f);
  }
}


cudaError_t launchAdjointStep(const AdjointStepArgs& A, cudaStream_t st) {
  if (A.n == 0) return cudaSuccess;
  if (A.entryStride == 0 || A.entryStride > 32) return cudaErrorInvalidValue;
  if (A.inCap > kGatherLanes * kGatherPerLane) return cudaErrorInvalidValue;
  const uint32_t blocks = (A.n + kAdjointThreads - 1) / kAdjointThreads;
  adjointStepKernel<<<blocks, kAdjointThreads, 0, st>>>(A);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  const uint32_t gatherBlocks = (uint32_t)(((size_t)A.n * kGatherLanes + kAdjointThreads - 1) / kAdjointThreads);
  adjointGatherKernel<<<gatherBlocks, kAdjointThreads, 0, st>>>(A);
  return cudaGetLastError();
}
cudaError_t launchFlockReduce(const FlockReduceArgs& A, cudaStream_t st) {
  if (A.nflocks == 0) return cudaSuccess;
  if (A.width < 1 || A.width > 3) return cudaErrorInvalidValue;
  flockReduceKernel<<<dim3(A.nflocks, kReduceParts), 256, 0, st>>>(A);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  flockReducePartsKernel<<<(A.nflocks * A.width + 255) / 256, 256, 0, st>>>(A);
  return cudaGetLastError();
}
cudaError_t launchLoss(const LossArgs& A, cudaStream_t st) {
  if (A.n == 0) return cudaSuccess;
  lossKernel<<<(A.n + 255) / 256, 256, 0, st>>>(A);
  return cudaGetLastError();
}
cudaError_t launchAdjointSeed(const SeedArgs& A, cudaStream_t st) {
  if (A.n == 0) return cudaSuccess;
  adjointSeedKernel<<<(A.n + 255) / 256, 256, 0, st>>>(A);
  return cudaGetLastError();
}
cudaError_t launchAdjointOut(const OutArgs& A, cudaStream_t st) {
  if (A.n == 0) return cudaSuccess;
  adjointOutKernel<<<(A.n + 255) / 256, 256, 0, st>>>(A);
  return cudaGetLastError();
}

}  // namespace brt
