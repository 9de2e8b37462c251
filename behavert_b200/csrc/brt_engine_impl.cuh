// brt_engine_impl.cuh -- the engine object shared by the host-side files of
// the library (brt_engine.cu, brt_adjoint_host.cu).  Not installed.
#pragma once

#include "brt_internal.cuh"
#include "brt_kernels.cuh"

#include <map>
#include <memory>
#include <tuple>
#include <vector>

namespace brt {
struct AdjointState;
void freeAdjoint(AdjointState* a);
}  // namespace brt

struct brt_engine {
  int device = 0;
  cudaStream_t stream = nullptr;
  uint32_t nflocks = 0, N = 0, C = 0, Cpad = 0, Mmax = 0, Fmax = 0, Fs = 0;
  std::vector<brt_params> params;
  std::vector<brt::FlockDev> flocksHost;
  brt::FlockDev* flocks = nullptr;
  uint32_t* agentBase = nullptr;
  float4* obstacles = nullptr;
  uint2* obsMask = nullptr;   // per-cell obstacle field (null when no flock has obstacles)
  bool anyKnn = false;
  bool school = false;        // the flocks use the Schooling law (schooling.mode 1 or 2)
  uint32_t* stepCounter = nullptr;  // device word: steps taken (keys the Schooling random stream)
  // device words of the cell-cull gate of scan variants 0 and 1: accumulator,
  // block ticket, and the result the flock kernel reads (nonzero: a sorted
  // position is NaN or outside the world, so cells are not culled)
  uint32_t* cullWords = nullptr;
  float4* membership[2] = {nullptr, nullptr};  // clusterMembership by agent id (ping-pong)
  int membershipCur = 0;
  bool forceTwoPass = false;  // option "two_pass": run the list-first kernel even when not needed
  // Launch options; the defaults are the autotuner's choice on both the
  // 1M-agent flock and the 1,024-flock batch.
  int phase2Variant = 2;      // option "phase2_variant": list walk shape (2: geometry, then features)
  int scanVariant = 5;        // option "scan_variant": neighbour-scan loop shape (5: warp-cooperative, windowed)
  // scan variant 6: the (flock, row segment) tiles of the staged tile kernel
  uint4* tiles = nullptr;
  uint32_t numTiles = 0;
  uint32_t* tileCounter = nullptr;
  uint32_t tileBlocks = 0;
  uint32_t fusedBlock = 64;   // option "block_size": threads per block of the single-pass flock kernel
  int regBudget = 64;         // option "registers" (or "wide_registers"): registers a thread of that kernel
  // state
  float4 *posA = nullptr, *fwdA = nullptr, *accA = nullptr, *posS = nullptr, *fwdS = nullptr, *accS = nullptr;
  float *featA = nullptr, *featS = nullptr;
  uint32_t *idA = nullptr, *idS = nullptr;
  float4* statsById = nullptr;
  float4* steer = nullptr;
  uint32_t* lists = nullptr;
  uint32_t listStride = 0;
  uint2* pairs[2] = {nullptr, nullptr};
  uint32_t *cellStart = nullptr, *cellEnd = nullptr;
  brt::SortPlan plan;
  void* sortMem = nullptr;
  brt::SortScratch ss;
  uint32_t* errWord = nullptr;
  // incremental re-sort (brt_resort.cu); option "incremental_sort"
  bool resortOn = true;
  brt::LookbackWait wait;  // bound of the look-back waits (copied into plan.wait)
  // A device check failed (a wait ran out, a pipeline invariant broke): the
  // slot order may no longer be a permutation.  brt_set_state rebuilds it.
  bool stateLost = false;
  uint32_t* resortMem = nullptr;   // one allocation carved into the arrays below
  size_t resortWords = 0;          // its size in words
  uint32_t *rsNewKey = nullptr, *rsPrefix = nullptr, *rsNext = nullptr, *rsBlockStay = nullptr;
  uint32_t *rsCount = nullptr, *rsHead = nullptr, *rsNewStart = nullptr, *rsTiles = nullptr;
  uint32_t *rsCounter = nullptr, *rsWords = nullptr, *rsStayBase = nullptr;
  float4* stage4 = nullptr;  // id-order staging (N float4)
  float* stageF = nullptr;   // id-order staging (N * Fmax)
  // pipeline state
  bool reordered = false, listsValid = false, recordLists = false;
  uint32_t finalPairs = 0;
  uint32_t paramsVersion = 0;
  std::map<std::tuple<uint32_t, uint32_t, bool, uint32_t>, cudaGraphExec_t> graphs;
  uint32_t smCount = 148;
  // per-stage timing: a ring of event sets, drained into totals
  static constexpr int kRing = 32;
  bool timing = false, capturing = false;
  cudaEvent_t ev[kRing][5] = {};
  bool pending[kRing] = {};
  int ringPos = 0;
  double stageMs[4] = {0, 0, 0, 0};
  uint64_t timedSteps = 0;
  // adjoint (brt_adjoint_host.cu): tape slot of the reorder's source slots
  uint32_t* tapePrev = nullptr;
  brt::AdjointState* adj = nullptr;
  bool adjointGraphs = true;  // option "adjoint_graphs"
  bool adjointExport = false; // option "adjoint_export"
  uint32_t weightsVersion = 0; // bumped by brt_set_steering_weights
  // registered per-agent arrays (brt_engine_add_array): `a` holds the array in
  // the engine's slot order, `s` is the gather target of each reorder (copied
  // back to `a`, so captured graphs always read and write the same buffers);
  // userIds is the agent id of each slot, permuted the same way.
  struct UserArray {
    uint32_t words = 0;
    uint32_t *a = nullptr, *s = nullptr;
  };
  std::vector<UserArray> user;
  UserArray userIds;
  uint32_t* userStage = nullptr;  // id-order staging, N * max words
  uint32_t userStageWords = 0;
  bool userFrozen = false;        // steps whose state is restored afterwards leave the arrays alone
};

namespace brt {

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

template <class T>
inline int devAlloc(T** p, size_t count) {
  *p = nullptr;
  if (count == 0) return BRT_OK;
  BRT_CUDA_TRY(cudaMalloc((void**)p, count * sizeof(T)));
  return BRT_OK;
}

// Defined in brt_engine.cu.
int engineEnqueueStep(brt_engine* e, float dt, bool record);
// The canonical arrays were overwritten: the next step runs the full sort.
cudaError_t engineInvalidateResort(brt_engine* e);
int engineSyncAndCheck(brt_engine* e);

}  // namespace brt
