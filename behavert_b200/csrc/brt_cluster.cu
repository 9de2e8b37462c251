// brt_cluster.cu -- BehaviorClustering analytics over the neighbour lists:
// cluster membership by local label propagation and the cluster hit rate
// (BehaviorClusteringPlugIn::computeClusterMembership / analyzeClusterHitRate,
// BehaviorClusteringPlugIn.h:828-894; kernels BehaviorClustering_kernel.cu
// :502-652).  The membership feature is a float4 per agent id: x the label,
// y the hit rate, z the mean label of the close neighbours (w unused), as the
// reference's float3 clusterMembership.  Labels are sorted slots (< 2^24, so
// exact as floats).  The reference's line-buffer connector for drawing the
// memberships (BehaviorClustering_CMConnection_kernel) is a graphics output
// and has no counterpart here.
#include "brt_agent.cuh"
#include "brt_kernels.cuh"

namespace brt {

// BehaviorClustering_resetClusterMembership_kernel (:640-660): every agent's
// label is its sorted slot.
__global__ void membershipResetKernel(ClusterArgs A) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const uint32_t id = __ldg(&A.idS[i]);
  float4 m = A.in[id];
  m.x = (float)i;
  A.out[id] = m;
}

// BehaviorClustering_computeClusterMembership_kernel (:588-632): one Jacobi
// sweep, label = min(own label, listed neighbours' labels).
__global__ void membershipSweepKernel(ClusterArgs A) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const uint32_t id = __ldg(&A.idS[i]);
  const float4 m = A.in[id];
  float lo = m.x;
  const uint32_t* lst = A.lists + (size_t)i * A.listStride;
  const uint32_t n = lst[0];
  for (uint32_t k = 0; k < n; ++k) {
    const float o = A.in[__ldg(&A.idS[lst[1 + k]])].x;
    if (lo > o) lo = o;
  }
  A.out[id] = make_float4(lo, m.y, m.z, m.w);
}

// BehaviorClustering_clusterHitRate (:502-583): among the listed neighbours
// closer than sameClusterMaxRadius, the fraction with the agent's label and
// their mean label (-1 with none).
__global__ void hitRateKernel(ClusterArgs A) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const uint32_t f = A.nflocks == 1 ? 0u : flockOfSlot(A.agentBase, A.nflocks, i);
  const FlockDev& fl = A.flocks[f];
  const uint32_t id = __ldg(&A.idS[i]);
  const float4 m = A.in[id];
  const float my = m.x;
  const AgentCtx a = makeCtx(__ldg(&A.posS[i]), make_float4(0.f, 0.f, 0.f, 0.f), fl);
  const uint32_t* lst = A.lists + (size_t)i * A.listStride;
  const uint32_t n = lst[0];
  int close = 0;
  float real = 0.0f, hit = 0.0f;
  for (uint32_t k = 0; k < n; ++k) {
    const uint32_t j = lst[1 + k];
    const float other = A.in[__ldg(&A.idS[j])].x;
    const f3 q = neighborImage(a, __ldg(&A.posS[j]), fl);
    const float dist = len3(sub3(q, a.pos));
    if (dist > A.radius) continue;
    ++close;
    real += other;
    if (my == other) hit += 1.0f;
  }
  if (close > 0) {
    hit /= (float)close;
    real /= (float)close;
  } else {
    real = -1.0f;
  }
  A.out[id] = make_float4(my, hit, real, m.w);
}

cudaError_t launchCluster(const ClusterArgs& A, int which, cudaStream_t st) {
  if (A.n == 0) return cudaSuccess;
  const uint32_t blocks = (A.n + 127) / 128;
  if (which == 0) membershipResetKernel<<<blocks, 128, 0, st>>>(A);
  else if (which == 1) membershipSweepKernel<<<blocks, 128, 0, st>>>(A);
  else hitRateKernel<<<blocks, 128, 0, st>>>(A);
  return cudaGetLastError();
}

}  // namespace brt
