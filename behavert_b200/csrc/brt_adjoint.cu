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
// slot (read coalesced, then zeroed so the buffer can take the next-earlier
// step's accumulation), and the adjoint of its input by canonical slot =
// the reorder's source slot `prev` of each sorted slot.  Neighbour
// contributions go into the input adjoint with float4 atomics; neighbours are
// near each other in both orders, so the atomics stay local in L2.
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

__device__ __forceinline__ void atomicAdd3(float4* dst, f3 v, float w) {
  atomicAdd(dst, make_float4(v.x, v.y, v.z, w));
}

// Per-flock FP64 sum of three values over a warp, then into `out`.
__device__ __forceinline__ void warpFlockSum3(double* out, uint32_t f, bool valid, double v0, double v1, double v2) {
  const uint32_t full = 0xFFFFFFFFu;
  const uint32_t f0 = __shfl_sync(full, f, 0);
  if (__all_sync(full, !valid || f == f0)) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      v0 += __shfl_down_sync(full, v0, o);
      v1 += __shfl_down_sync(full, v1, o);
      v2 += __shfl_down_sync(full, v2, o);
    }
    if ((threadIdx.x & 31u) == 0u) {
      atomicAdd(&out[3 * f0 + 0], v0);
      atomicAdd(&out[3 * f0 + 1], v1);
      atomicAdd(&out[3 * f0 + 2], v2);
    }
  } else if (valid) {
    atomicAdd(&out[3 * f + 0], v0);
    atomicAdd(&out[3 * f + 1], v1);
    atomicAdd(&out[3 * f + 2], v2);
  }
}

}  // namespace

// Branch bits of the exported flag word (the oracle's frozen-branch layout).
constexpr uint32_t kBrLow = 1u, kBrLimited = 2u, kBrClipF = 4u, kBrClipV = 8u;

__global__ void __launch_bounds__(kAdjointThreads) adjointStepKernel(AdjointStepArgs A) {
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

    // The adjoint of this step's output; the buffers are zeroed for the
    // accumulation of the next-earlier step.
    const float4 gOp = A.gOutP[i], gOf = A.gOutF[i], gOa = A.gOutA[i];
    A.gOutP[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    A.gOutF[i] = make_float4(0.f, 0.f, 0.f, 0.f);

    // --- forward recomputation (flockingSteer's sequence) -----------------
    f3 sSep = mk3(0.f, 0.f, 0.f), sAli = mk3(0.f, 0.f, 0.f), sCoh = mk3(0.f, 0.f, 0.f);
    uint32_t cSep = 0, cAli = 0, cCoh = 0, mS = 0, mA = 0, mC = 0;
    for (uint32_t k = 0; k < n; ++k) {
      const uint32_t j = lst[1 + k];
      const f3 other = neighborImage(a, __ldg(&A.posS[j]), fl);
      const f3 offset = sub3(other, a.pos);
      const float d2 = dot3(offset, offset);
      const float dist = sqrtf(d2);
      const f3 nrm = mul3(offset, 1.0f / dist);
      const float cosAngle = dot3(a.fwd, nrm);
      if (inBoid(dist, cosAngle, fl.minR, fl.sep[1], fl.sep[2])) {
        sSep = add3(sSep, div3(offset, -d2));
        ++cSep;
        mS |= 1u << k;
      }
      if (inBoid(dist, cosAngle, fl.minR, fl.ali[1], fl.ali[2])) {
        sAli = add3(sAli, xyz(__ldg(&A.fwdS[j])));
        ++cAli;
        mA |= 1u << k;
      }
      if (inBoid(dist, cosAngle, fl.minR, fl.coh[1], fl.coh[2])) {
        sCoh = add3(sCoh, other);
        ++cCoh;
        mC |= 1u << k;
      }
    }
    const float w[3] = {fl.sep[0], fl.ali[0], fl.coh[0]};
    f3 x[3], u[3];
    const uint32_t cnt[3] = {cSep, cAli, cCoh};
    x[0] = cSep ? div3(sSep, (float)cSep) : sSep;
    x[1] = cAli ? sub3(div3(sAli, (float)cAli), a.fwd) : sAli;
    x[2] = cCoh ? sub3(div3(sCoh, (float)cCoh), a.pos) : sCoh;
    f3 steer = mk3(0.f, 0.f, 0.f);
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      u[b] = cnt[b] ? normalize3(x[b]) : x[b];
      if (w[b] != 0.0f) steer = add3(mul3(u[b], w[b]), steer);
    }
    if (fl.numObstacles && fl.obsW != 0.0f) steer = obstacleSteer(a, fl, A.obstacles, A.obsMask, steer);

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
        cosine = 1.0f + ((-1.0f - 1.0f) * powf(range, 20.0f));
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
      const f3 v = add3(mul3(fwd, speed), mul3(smoothed, dt));
      if (!(len3(v) <= maxS)) br |= kBrClipV;
      const f3 vT = truncateLength(v, maxS);

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
        selfS += gC * (-40.0f * powf(range, 19.0f) / s0);
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
      gw[b] = dot3(gSteer, u[b]);
      gx[b] = normalizeBar(x[b], mul3(gSteer, w[b]));
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
    const uint32_t any = mS | mA | mC;
    for (uint32_t k = 0; k < n; ++k) {
      if (!((any >> k) & 1u)) continue;
      const uint32_t j = lst[1 + k];
      const uint32_t tj = __ldg(&A.prev[j]);
      f3 gp = mk3(0.f, 0.f, 0.f);
      if ((mS >> k) & 1u) {
        // -o / |o|^2 with Jacobian -(I / d2 - 2 o o^T / d2^2)
        const f3 other = neighborImage(a, __ldg(&A.posS[j]), fl);
        const f3 o = sub3(other, a.pos);
        const float d2 = dot3(o, o);
        const f3 go = mul3(sub3(div3(gSs, d2), mul3(o, 2.0f * dot3(o, gSs) / (d2 * d2))), -1.0f);
        gp = add3(gp, go);
        selfP = sub3(selfP, go);
      }
      if ((mC >> k) & 1u) gp = add3(gp, gSc);
      if (((mS | mC) >> k) & 1u) atomicAdd3(&A.gInP[tj], gp, 0.0f);
      if ((mA >> k) & 1u) atomicAdd3(&A.gInF[tj], gSa, 0.0f);
    }
    atomicAdd3(&A.gInP[self], selfP, 0.0f);
    atomicAdd3(&A.gInF[self], selfF, selfS);
    A.gInA[self] = make_float4(selfA.x, selfA.y, selfA.z, 0.0f);

    if (A.exportFlags) {
      const uint32_t id = __ldg(&A.idS[i]);
      reinterpret_cast<uint4*>(A.exportFlags)[id] = make_uint4(br, mS, mA, mC);
      uint32_t* row = A.exportLists + (size_t)id * A.listStride;
      row[0] = n;
      for (uint32_t k = 0; k < n; ++k) row[1 + k] = __ldg(&A.idS[lst[1 + k]]);
    }
  }
  warpFlockSum3(A.gW, f, valid, (double)gw[0], (double)gw[1], (double)gw[2]);
}

// Loss = sum over flocks of the mean squared minimum-image distance between
// final and target positions (FP64), per flock into lossPerFlock, and the
// unscaled terminal position adjoint 2 d / n_f (canonical order).
__global__ void __launch_bounds__(256) lossKernel(LossArgs A) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < A.n;
  uint32_t f = 0;
  double l = 0.0;
  if (valid) {
    f = A.nflocks == 1 ? 0u : flockOfSlot(A.agentBase, A.nflocks, i);
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
    l = (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) * inv;
    A.gT[i] = make_float4((float)(2.0 * d[0] * inv), (float)(2.0 * d[1] * inv), (float)(2.0 * d[2] * inv), 0.0f);
  }
  const uint32_t full = 0xFFFFFFFFu;
  const uint32_t f0 = __shfl_sync(full, f, 0);
  if (__all_sync(full, !valid || f == f0)) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(full, l, o);
    if ((threadIdx.x & 31u) == 0u) atomicAdd(&A.lossPerFlock[f0], l);
  } else if (valid) {
    atomicAdd(&A.lossPerFlock[f], l);
  }
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
  adjointStepKernel<<<(A.n + kAdjointThreads - 1) / kAdjointThreads, kAdjointThreads, 0, st>>>(A);
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
