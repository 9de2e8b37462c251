// brt_school.cu -- the Schooling plugin's steering law (Couzin-style zones)
// in the fused step and as the reference's stage-wise functionalities.
//
// Fused: one thread per sorted slot scans the 27 neighbour cells into a
// shared-memory list (the same scan as the flocking kernel), then applies
//   mode 1, Schooling_animateSchool (Schooling_kernel.cu:226-318), or
//   mode 2, Schooling_repulsion -> Schooling_attractionOrientation ->
//           Schooling_move (Schooling_kernel.cu:64-221),
// and writes the new state at the same slot.  Stage-wise kernels reproduce
// each reference kernel over the lists of brt_compute_neighborhoods, with
// the steering force in the engine's steer buffer.
//
// Periodic world: the reference's boundary term (steer back toward the
// centre when outside the box) is the identity, and positions are wrapped
// after the move.  The random deviation uses a counter-based generator keyed
// on (seed, step, agent id) in place of the reference's Mersenne Twister.
#include "brt_agent.cuh"
#include "brt_kernels.cuh"

namespace brt {

// splitmix64 (Steele, Lea, Flood, "Fast splittable pseudorandom number
// generators", 2014).
__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  uint64_t z = x + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Three uniform values in [0, 1) with 24 random bits each (exact floats).
__device__ __forceinline__ f3 schoolRandom(uint32_t seed, uint32_t step, uint32_t id) {
  const uint64_t base = splitmix64(((uint64_t)seed << 32) | step);
  const uint64_t u1 = splitmix64(base ^ (uint64_t)id);
  const uint64_t u2 = splitmix64(u1);
  const float k = 5.9604644775390625e-08f;  // 2^-24
  return mk3((float)(uint32_t)(u1 >> 40) * k, (float)(uint32_t)((u1 >> 16) & 0xFFFFFFu) * k,
             (float)(uint32_t)(u2 >> 40) * k);
}

// Sum of unit offsets toward listed neighbours closer than r_r
// (Schooling_kernel.cu:75-86 and 240-253).
__device__ __forceinline__ f3 schoolRepulsion(const AgentCtx& a, const FlockDev& fl, const uint32_t* list, uint32_t ls,
                                              uint32_t n, const float4* __restrict__ posS, uint32_t& found) {
  f3 s = mk3(0.f, 0.f, 0.f);
  found = 0;
  for (uint32_t k = 0; k < n; ++k) {
    const f3 other = neighborImage(a, __ldg(&posS[list[k * ls]]), fl);
    const f3 off = sub3(other, a.pos);
    const float dist = len3(off);
    if (dist < fl.schRr) {
      s = add3(s, div3(off, len3(off)));
      ++found;
    }
  }
  return s;
}

// attraction * w_a + orientation * w_o over the listed neighbours in the
// zone: dist < r_p (animateSchool, :259-279), or the zone of
// inAttractionOrientationZone with the blind angle (Schooling_resources.cu
// :34-71, dist <= r_p and cos > eta).
__device__ __forceinline__ f3 schoolAttractOrient(const AgentCtx& a, const FlockDev& fl, const uint32_t* list, uint32_t ls,
                                                  uint32_t n, const float4* __restrict__ posS,
                                                  const float4* __restrict__ fwdS, bool blind) {
  f3 orient = div3(a.fwd, len3(a.fwd));
  f3 attr = mk3(0.f, 0.f, 0.f);
  for (uint32_t k = 0; k < n; ++k) {
    const uint32_t j = list[k * ls];
    const f3 other = neighborImage(a, __ldg(&posS[j]), fl);
    const f3 off = sub3(other, a.pos);
    const float dist = len3(off);
    const bool in = blind ? (!(dist > fl.schRp) && dot3(a.fwd, normalize3(off)) > fl.schEta) : (dist < fl.schRp);
    if (in) {
      attr = add3(attr, div3(off, len3(off)));
      const f3 wj = xyz(__ldg(&fwdS[j]));
      orient = add3(orient, div3(wj, len3(wj)));
    }
  }
  return add3(mul3(attr, fl.schWa), mul3(orient, fl.schWo));
}

// The repulsion stage's force (Schooling_repulsion): -normalize(sum) when
// the sum is nonzero.
__device__ __forceinline__ f3 repulsionForce(f3 s) {
  if (len3(s) > 0.0f) {
    const f3 u = normalize3(s);
    return mk3(-u.x, -u.y, -u.z);
  }
  return s;
}

// Schooling_attractionOrientation: keep a nonzero repulsion force, else the
// normalised attraction/orientation blend.
__device__ __forceinline__ f3 attractionOrientationForce(const AgentCtx& a, const FlockDev& fl, f3 steer, const uint32_t* list,
                                                         uint32_t ls, uint32_t n, const float4* __restrict__ posS,
                                                         const float4* __restrict__ fwdS) {
  if (len3(steer) > 0.0f) return steer;
  f3 nf = schoolAttractOrient(a, fl, list, ls, n, posS, fwdS, true);
  if (len3(nf) > 0.0f) nf = normalize3(nf);
  return nf;
}

// Schooling_move (:131-221): random deviation, turn limit, constant-speed
// step of s * forward * 0.2.
__device__ __forceinline__ Integrated schoolMove(const AgentCtx& a, const FlockDev& fl, f3 nf, uint32_t id, uint32_t step,
                                                 float4 acc4) {
  if (fl.schRand > 0.0f) {
    const f3 r = schoolRandom(fl.schSeed, step, id);
    const float w = fl.schRand;
    const f3 rd = sub3(mul3(mul3(r, w), 2.0f), mul3(mk3(1.0f, 1.0f, 1.0f), w));
    nf = normalize3(add3(nf, rd));
  }
  const f3 fwd = vecLimitDeviationAngle(nf, fl.schTheta, a.fwd);
  f3 pos = add3(a.pos, mul3(mul3(fwd, fl.schS), 0.2f));
  if (fl.use2D) pos.y = 0.5f;
  Integrated r;
  r.pos = make_float4(wrapPeriodic(pos.x, fl.L), wrapPeriodic(pos.y, fl.L), wrapPeriodic(pos.z, fl.L), 1.0f);
  r.fwd = make_float4(fwd.x, fwd.y, fwd.z, fl.schS);
  r.acc = acc4;
  return r;
}

// Schooling_animateSchool (:226-318).
__device__ __forceinline__ Integrated animateSchool(const AgentCtx& a, const FlockDev& fl, const uint32_t* list, uint32_t ls,
                                                    uint32_t n, const float4* __restrict__ posS,
                                                    const float4* __restrict__ fwdS, float4 acc4) {
  uint32_t found = 0;
  f3 nf = schoolRepulsion(a, fl, list, ls, n, posS, found);
  nf = mk3(-nf.x, -nf.y, -nf.z);
  if (found == 0) nf = schoolAttractOrient(a, fl, list, ls, n, posS, fwdS, false);
  if (fl.use2D) nf.y = 0.0f;
  if (len3(nf) > 0.0f) nf = normalize3(nf);
  const f3 fwd = vecLimitDeviationAngle(nf, fl.schTheta, a.fwd);
  f3 pos = add3(a.pos, mul3(mul3(fwd, fl.schS), 0.1f));
  if (fl.use2D) pos.y = 0.5f;
  Integrated r;
  r.pos = make_float4(wrapPeriodic(pos.x, fl.L), wrapPeriodic(pos.y, fl.L), wrapPeriodic(pos.z, fl.L), 1.0f);
  r.fwd = make_float4(fwd.x, fwd.y, fwd.z, fl.schS);
  r.acc = acc4;
  return r;
}

__device__ __forceinline__ void copyFeatures(const float* featS, float* featA, uint32_t Fs, uint32_t i) {
  if (!Fs) return;
  const float4* src = reinterpret_cast<const float4*>(featS) + (size_t)i * (Fs / 4);
  float4* dst = reinterpret_cast<float4*>(featA) + (size_t)i * (Fs / 4);
  for (uint32_t q = 0; q < Fs / 4; ++q) dst[q] = __ldg(&src[q]);
}

// The lists come from the warp-cooperative windowed scan (the flock
// kernel's scan 5): every lane of a warp takes part, inactive lanes mirror
// the last agent read-only and leave after the scan.
__global__ void __launch_bounds__(128) schoolKernel(FusedArgs A) {
  extern __shared__ uint32_t sList[];
  const uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = i0 < A.n;
  const uint32_t i = active ? i0 : A.n - 1;
  const uint32_t f = A.nflocks == 1 ? 0u : flockOfSlot(A.agentBase, A.nflocks, i);
  const FlockDev& fl = A.flocks[f];
  const float4 p4 = __ldg(&A.posS[i]);
  const f3 p = xyz(p4);
  const uint32_t G = fl.G;
  const uint32_t key = fl.cellBase + ((uint32_t)gridCoord(p.z, fl) * G + (uint32_t)gridCoord(p.y, fl)) * G +
                       (uint32_t)gridCoord(p.x, fl);
  const uint32_t ls = blockDim.x + 1;  // odd: one vote's rows fall in distinct banks
  const uint32_t n = scanNeighborsCooperative<kCoopCachedRounds, kCoopWindowAgents>(
      active, i, p, key, A.flocks, f, A.cellStart, A.cellEnd, A.posS, sList, ls, threadIdx.x & ~31u);
  if (!active) return;
  uint32_t* list = sList + threadIdx.x;
  const float4 w4 = __ldg(&A.fwdS[i]), a4 = __ldg(&A.accS[i]);
  if (A.lists) {
    uint32_t* out = A.lists + (size_t)i * A.listStride;
    out[0] = n;
    for (uint32_t k = 0; k < n; ++k) out[1 + k] = list[k * ls];
  }
  const AgentCtx a = makeCtx(p4, w4, fl);
  const uint32_t id = __ldg(&A.idS[i]);
  Integrated r;
  if (fl.school == 1) {
    r = animateSchool(a, fl, list, ls, n, A.posS, A.fwdS, a4);
  } else {
    uint32_t found = 0;
    f3 steer = repulsionForce(schoolRepulsion(a, fl, list, ls, n, A.posS, found));
    steer = attractionOrientationForce(a, fl, steer, list, ls, n, A.posS, A.fwdS);
    r = schoolMove(a, fl, steer, id, A.stepCounter ? *A.stepCounter : 0u, a4);
  }
  A.posA[i] = r.pos;
  A.fwdA[i] = r.fwd;
  A.accA[i] = r.acc;
  A.idA[i] = id;
  copyFeatures(A.featS, A.featA, A.Fs, i);
}

// Stage-wise: which = 0 repulsion, 1 attraction/orientation (both into the
// steer buffer), 2 move, 3 animateSchool (both write the new state).
__global__ void __launch_bounds__(128) schoolStageKernel(StageArgs A, int which) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const uint32_t f = A.nflocks == 1 ? 0u : flockOfSlot(A.agentBase, A.nflocks, i);
  const FlockDev& fl = A.flocks[f];
  const uint32_t* lst = A.lists + (size_t)i * A.listStride;
  const uint32_t n = lst[0];
  const float4 p4 = __ldg(&A.posS[i]), w4 = __ldg(&A.fwdS[i]), a4 = __ldg(&A.accS[i]);
  const AgentCtx a = makeCtx(p4, w4, fl);
  if (which == 0) {
    uint32_t found = 0;
    const f3 s = repulsionForce(schoolRepulsion(a, fl, lst + 1, 1, n, A.posS, found));
    A.steer[i] = make_float4(s.x, s.y, s.z, 0.0f);
    return;
  }
  if (which == 1) {
    const f3 s = attractionOrientationForce(a, fl, xyz(A.steer[i]), lst + 1, 1, n, A.posS, A.fwdS);
    A.steer[i] = make_float4(s.x, s.y, s.z, 0.0f);
    return;
  }
  const uint32_t id = __ldg(&A.idS[i]);
  const Integrated r = which == 2 ? schoolMove(a, fl, xyz(A.steer[i]), id, A.stepCounter ? *A.stepCounter : 0u, a4)
                                  : animateSchool(a, fl, lst + 1, 1, n, A.posS, A.fwdS, a4);
  A.posA[i] = r.pos;
  A.fwdA[i] = r.fwd;
  A.accA[i] = r.acc;
  A.idA[i] = id;
  copyFeatures(A.featS, A.featA, A.Fs, i);
}

cudaError_t launchSchool(const FusedArgs& A, cudaStream_t st) {
  if (A.n == 0) return cudaSuccess;
  const uint32_t block = 128;
  schoolKernel<<<(A.n + block - 1) / block, block, (size_t)(block + 1) * A.Mmax * 4, st>>>(A);
  return cudaGetLastError();
}

cudaError_t launchSchoolStage(const StageArgs& A, int which, cudaStream_t st) {
  if (A.n == 0) return cudaSuccess;
  schoolStageKernel<<<(A.n + 127) / 128, 128, 0, st>>>(A, which);
  return cudaGetLastError();
}

cudaError_t configureSchoolKernels(uint32_t Mmax) {
  return cudaFuncSetAttribute(schoolKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(129 * Mmax * 4));
}

}  // namespace brt
