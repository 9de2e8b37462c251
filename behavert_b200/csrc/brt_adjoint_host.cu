// brt_adjoint_host.cu -- host side of the differentiable rollout (no
// reference counterpart).
//
// brt_adjoint_forward runs T fused steps from the engine's current state,
// keeping a checkpoint of the canonical state every k steps, then evaluates
// the FP64 loss against id-ordered targets.  brt_adjoint_backward walks the
// checkpoints from last to first: it restores one, re-runs its (up to) k
// steps -- hash, sort, reorder and the fused pass, exactly as in the forward
// -- with the reorder's sorted state, source slots and neighbour lists
// written into a k-step tape, then runs the reverse kernel over the tape
// from its last step to its first.  Both directions are captured as CUDA
// graphs (cached by T, k, dt and the parameter version), so a whole forward
// or backward is one graph launch.  The engine's state after the backward is
// the final state of the forward.
#include "brt_engine_impl.cuh"

#include <cstring>
#include <string>

namespace brt {

void setLastError(const std::string& msg);

struct AdjointState {
  uint32_t T = 0, k = 0, nck = 0;
  float dt = 0.0f;
  bool taped = false;
  uint32_t version = 0;       // engine paramsVersion of the taped forward
  uint32_t weightsVersion = 0;
  uint32_t capCk = 0, capK = 0, capExport = 0;
  std::vector<void*> mem;
  // checkpoints (nck x N) and the saved final state
  float4 *ckPos = nullptr, *ckFwd = nullptr, *ckAcc = nullptr;
  uint32_t* ckId = nullptr;
  float4 *finPos = nullptr, *finFwd = nullptr, *finAcc = nullptr;
  uint32_t* finId = nullptr;
  float* finFeat = nullptr;
  // two k-step tapes: the backward recomputes segment c - 1 into one while
  // the reverse of segment c reads the other
  struct Tape {
    float4 *pos = nullptr, *fwd = nullptr, *acc = nullptr;
    uint32_t *prev = nullptr, *id = nullptr, *lists = nullptr;
  } tape[2];
  // the reverse chain's stream and the events that order it against the
  // recompute chain on the engine stream (2 per checkpoint segment)
  cudaStream_t revStream = nullptr;
  std::vector<cudaEvent_t> events;
  // adjoint buffers
  float4* g[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
  float4* gT = nullptr;
  float4* target = nullptr;
  float4* io[4] = {nullptr, nullptr, nullptr, nullptr};  // id-order staging in / out
  double* gW = nullptr;
  double* loss = nullptr;
  float* scale = nullptr;
  uint32_t *expLists = nullptr, *expFlags = nullptr;
  float4* expState = nullptr;  // per step: input pos, fwd, acc by agent id
  // emit -> gather hand-over of one reverse step, and the weight sums
  float4 *contrib = nullptr, *selfP = nullptr, *selfF = nullptr;
  double* partial = nullptr;  // per-flock reduction parts
  uint32_t *inCount = nullptr, *ovHead = nullptr, *ovNext = nullptr;
  float4* inbox = nullptr;
  uint32_t inCap = 0;
  double* accW = nullptr;
  // graphs: (kind, T, k, dt bits, params version, variant bits)
  std::map<std::tuple<int, uint32_t, uint32_t, uint32_t, uint32_t, uint32_t>, cudaGraphExec_t> graphs;
};

void freeAdjoint(AdjointState* a) {
  if (!a) return;
  for (auto& kv : a->graphs) cudaGraphExecDestroy(kv.second);
  for (void* p : a->mem) cudaFree(p);
  for (cudaEvent_t ev : a->events) cudaEventDestroy(ev);
  if (a->revStream) cudaStreamDestroy(a->revStream);
  delete a;
}

namespace {

template <class T>
int adjAlloc(AdjointState* a, T** p, size_t count) {
  int rc = devAlloc(p, std::max<size_t>(count, 1));
  if (!rc) a->mem.push_back(*p);
  return rc;
}

void dropGraphs(AdjointState* a) {
  for (auto& kv : a->graphs) cudaGraphExecDestroy(kv.second);
  a->graphs.clear();
}

// The reverse kernels cover the flocking, obstacle and integration terms.
int checkSupported(brt_engine* e) {
  for (const FlockDev& d : e->flocksHost) {
    if (d.useKnn) { setLastError("adjoint: kNN neighbour lists are not supported"); return BRT_ERR_CONFIG; }
    if (d.use2D) { setLastError("adjoint: use2DProjection is not supported"); return BRT_ERR_CONFIG; }
    if (d.school) { setLastError("adjoint: the Schooling law is not supported"); return BRT_ERR_CONFIG; }
    if (d.F > 0 && (d.clus != 0.0f || d.aclus != 0.0f)) {
      setLastError("adjoint: feature clustering steering is not supported");
      return BRT_ERR_CONFIG;
    }
  }
  if (e->Mmax > 32) { setLastError("adjoint: maxNeighbors must be <= 32"); return BRT_ERR_CONFIG; }
  if (e->forceTwoPass) { setLastError("adjoint: option two_pass must be off"); return BRT_ERR_CONFIG; }
  return BRT_OK;
}

// (Re)allocates the checkpoint and tape storage for nck checkpoints and k
// tape steps; buffers only grow.
int ensureCapacity(brt_engine* e, uint32_t nck, uint32_t k, uint32_t T) {
  AdjointState* a = e->adj;
  const size_t n = e->N;
  int rc = BRT_OK;
  bool changed = false;
  if (a->mem.empty()) {
    changed = true;
    for (int s = 0; s < 2; ++s)
      for (int c = 0; c < 3; ++c) if ((rc = adjAlloc(a, &a->g[s][c], n))) return rc;
    if ((rc = adjAlloc(a, &a->gT, n))) return rc;
    if ((rc = adjAlloc(a, &a->target, n))) return rc;
    for (int c = 0; c < 4; ++c) if ((rc = adjAlloc(a, &a->io[c], n))) return rc;
    if ((rc = adjAlloc(a, &a->gW, 3 * (size_t)e->nflocks))) return rc;
    if ((rc = adjAlloc(a, &a->loss, e->nflocks))) return rc;
    if ((rc = adjAlloc(a, &a->scale, e->nflocks))) return rc;
    if ((rc = adjAlloc(a, &a->finPos, n))) return rc;
    if ((rc = adjAlloc(a, &a->finFwd, n))) return rc;
    if ((rc = adjAlloc(a, &a->finAcc, n))) return rc;
    if ((rc = adjAlloc(a, &a->finId, n))) return rc;
    if ((rc = adjAlloc(a, &a->finFeat, n * e->Fs))) return rc;
    if ((rc = adjAlloc(a, &a->contrib, 2 * n * (size_t)e->Mmax))) return rc;
    if ((rc = adjAlloc(a, &a->selfP, n))) return rc;
    if ((rc = adjAlloc(a, &a->selfF, n))) return rc;
    if ((rc = adjAlloc(a, &a->partial, 3 * (size_t)kReduceParts * e->nflocks))) return rc;
    // in-degree is about the list length: room for twice maxNeighbors, the
    // rest overflows into a linked list
    a->inCap = std::min(64u, 2u * e->Mmax);
    if ((rc = adjAlloc(a, &a->inCount, n))) return rc;
    if ((rc = adjAlloc(a, &a->inbox, 2 * n * (size_t)a->inCap))) return rc;
    if ((rc = adjAlloc(a, &a->ovHead, n))) return rc;
    if ((rc = adjAlloc(a, &a->ovNext, n * (size_t)e->Mmax))) return rc;
    if ((rc = adjAlloc(a, &a->accW, 3 * n))) return rc;
    BRT_CUDA_TRY(cudaMemsetAsync(a->target, 0, n * 16, e->stream));
  }
  auto regrow = [&](auto** p, size_t count) -> int {
    for (auto it = a->mem.begin(); it != a->mem.end(); ++it)
      if (*it == (void*)*p) { cudaFree(*it); a->mem.erase(it); break; }
    *p = nullptr;
    return adjAlloc(a, p, count);
  };
  if (nck > a->capCk) {
    BRT_CUDA_TRY(cudaStreamSynchronize(e->stream));
    if ((rc = regrow(&a->ckPos, n * nck)) || (rc = regrow(&a->ckFwd, n * nck)) || (rc = regrow(&a->ckAcc, n * nck)) ||
        (rc = regrow(&a->ckId, n * nck)))
      return rc;
    a->capCk = nck;
    changed = true;
  }
  if (k > a->capK) {
    BRT_CUDA_TRY(cudaStreamSynchronize(e->stream));
    for (auto& t : a->tape)
      if ((rc = regrow(&t.pos, n * k)) || (rc = regrow(&t.fwd, n * k)) || (rc = regrow(&t.acc, n * k)) ||
          (rc = regrow(&t.prev, n * k)) || (rc = regrow(&t.id, n * k)) || (rc = regrow(&t.lists, n * k * e->listStride)))
        return rc;
    a->capK = k;
    changed = true;
  }
  if (!a->revStream) BRT_CUDA_TRY(cudaStreamCreateWithFlags(&a->revStream, cudaStreamNonBlocking));
  while (a->events.size() < 2 * (size_t)nck) {
    cudaEvent_t ev = nullptr;
    BRT_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    a->events.push_back(ev);
  }
  if (e->adjointExport && T > a->capExport) {
    BRT_CUDA_TRY(cudaStreamSynchronize(e->stream));
    if ((rc = regrow(&a->expLists, n * T * e->listStride)) || (rc = regrow(&a->expFlags, n * T * 4)) ||
        (rc = regrow(&a->expState, n * T * 3)))
      return rc;
    a->capExport = T;
    changed = true;
  }
  if (changed) dropGraphs(a);
  return BRT_OK;
}

int copyState(brt_engine* e, float4* pos, float4* fwd, float4* acc, uint32_t* id, const float4* spos, const float4* sfwd,
              const float4* sacc, const uint32_t* sid) {
  const size_t n = e->N;
  BRT_CUDA_TRY(cudaMemcpyAsync(pos, spos, n * 16, cudaMemcpyDeviceToDevice, e->stream));
  BRT_CUDA_TRY(cudaMemcpyAsync(fwd, sfwd, n * 16, cudaMemcpyDeviceToDevice, e->stream));
  BRT_CUDA_TRY(cudaMemcpyAsync(acc, sacc, n * 16, cudaMemcpyDeviceToDevice, e->stream));
  BRT_CUDA_TRY(cudaMemcpyAsync(id, sid, n * 4, cudaMemcpyDeviceToDevice, e->stream));
  // a checkpoint restored into the engine: its order is not the last step's
  if (pos == e->posA) BRT_CUDA_TRY(engineInvalidateResort(e));
  return BRT_OK;
}

// The taped forward: checkpoints, steps, final state, loss.
int enqueueForward(brt_engine* e) {
  AdjointState* a = e->adj;
  const size_t n = e->N;
  int rc = BRT_OK;
  for (uint32_t c = 0; c < a->nck; ++c) {
    if ((rc = copyState(e, a->ckPos + c * n, a->ckFwd + c * n, a->ckAcc + c * n, a->ckId + c * n, e->posA, e->fwdA,
                        e->accA, e->idA)))
      return rc;
    const uint32_t steps = std::min(a->k, a->T - c * a->k);
    for (uint32_t s = 0; s < steps; ++s)
      if ((rc = engineEnqueueStep(e, a->dt, false))) return rc;
  }
  if ((rc = copyState(e, a->finPos, a->finFwd, a->finAcc, a->finId, e->posA, e->fwdA, e->accA, e->idA))) return rc;
  if (e->Fs) BRT_CUDA_TRY(cudaMemcpyAsync(a->finFeat, e->featA, n * e->Fs * 4, cudaMemcpyDeviceToDevice, e->stream));
  LossArgs L;
  std::memset(&L, 0, sizeof(L));
  L.posA = e->posA; L.idA = e->idA; L.target = a->target;
  L.flocks = e->flocks; L.agentBase = e->agentBase; L.nflocks = e->nflocks; L.n = e->N;
  L.lossTerm = a->accW; L.gT = a->gT;  // accW is free until the backward
  BRT_CUDA_TRY(launchLoss(L, e->stream));
  FlockReduceArgs R;
  R.vals = a->accW; R.width = 1; R.agentBase = e->agentBase; R.nflocks = e->nflocks; R.out = a->loss;
  R.partial = a->partial;
  BRT_CUDA_TRY(launchFlockReduce(R, e->stream));
  return BRT_OK;
}

// Re-runs one segment's steps with a tape as the step's sorted-state and
// list buffers.
int enqueueRecompute(brt_engine* e, uint32_t steps, const AdjointState::Tape& tp) {
  AdjointState* a = e->adj;
  const size_t n = e->N;
  float4 *posS = e->posS, *fwdS = e->fwdS, *accS = e->accS;
  uint32_t *idS = e->idS, *lists = e->lists;
  // the engine returns to the forward's final state afterwards, so
  // registered arrays (already at that state) are not permuted again
  const bool wasFrozen = e->userFrozen;
  e->userFrozen = true;
  int rc = BRT_OK;
  for (uint32_t s = 0; s < steps && !rc; ++s) {
    e->posS = tp.pos + s * n; e->fwdS = tp.fwd + s * n; e->accS = tp.acc + s * n;
    e->idS = tp.id + s * n;
    e->lists = tp.lists + s * n * e->listStride;
    e->tapePrev = tp.prev + s * n;
    rc = engineEnqueueStep(e, a->dt, true);
  }
  e->posS = posS; e->fwdS = fwdS; e->accS = accS; e->idS = idS; e->lists = lists;
  e->tapePrev = nullptr;
  e->userFrozen = wasFrozen;
  return rc;
}

// variant bits: 1 extra position adjoint, 2 extra forward adjoint, 4 extra
// acceleration adjoint, 8 per-flock loss scale, 16 tape export.
int enqueueBackward(brt_engine* e, uint32_t variant) {
  AdjointState* a = e->adj;
  const size_t n = e->N;
  int rc = BRT_OK;
  SeedArgs S;
  std::memset(&S, 0, sizeof(S));
  S.gT = a->gT;
  S.scale = (variant & 8u) ? a->scale : nullptr;
  S.extraP = (variant & 1u) ? a->io[0] : nullptr;
  S.extraF = (variant & 2u) ? a->io[1] : nullptr;
  S.extraA = (variant & 4u) ? a->io[2] : nullptr;
  S.idA = a->finId; S.agentBase = e->agentBase; S.nflocks = e->nflocks; S.n = e->N;
  int cur = 0;
  S.gP = a->g[cur][0]; S.gF = a->g[cur][1]; S.gA = a->g[cur][2];
  BRT_CUDA_TRY(launchAdjointSeed(S, e->stream));
  BRT_CUDA_TRY(cudaMemsetAsync(a->accW, 0, 24 * n, e->stream));
  BRT_CUDA_TRY(cudaMemsetAsync(a->inCount, 0, 4 * n, e->stream));     // empty in-lists
  BRT_CUDA_TRY(cudaMemsetAsync(a->ovHead, 0xFF, 4 * n, e->stream));    // kNoEntry
  // Two chains: the recompute of each checkpoint segment on the engine
  // stream (it owns the engine's buffers) and the reverse steps on revStream.
  // Segment c's reverse waits for its recompute; the recompute of c - 1 runs
  // beside it into the other tape, once the reverse of c + 1 (the last
  // reader of that tape) is done.  Both are latency-bound at these sizes, so
  // the two overlap on the GPU; the results are those of running them in
  // sequence.
  cudaStream_t rs = a->revStream;
  auto evRecomputed = [a](int c) { return a->events[2 * (size_t)c]; };
  auto evReversed = [a](int c) { return a->events[2 * (size_t)c + 1]; };
  auto recompute = [&](int c) -> int {
    if (c + 2 < (int)a->nck) BRT_CUDA_TRY(cudaStreamWaitEvent(e->stream, evReversed(c + 2), 0));
    int r = copyState(e, e->posA, e->fwdA, e->accA, e->idA, a->ckPos + c * n, a->ckFwd + c * n, a->ckAcc + c * n,
                      a->ckId + c * n);
    if (r) return r;
    const uint32_t steps = std::min(a->k, a->T - (uint32_t)c * a->k);
    if ((r = enqueueRecompute(e, steps, a->tape[c & 1]))) return r;
    BRT_CUDA_TRY(cudaEventRecord(evRecomputed(c), e->stream));
    return BRT_OK;
  };
  if ((rc = recompute((int)a->nck - 1))) return rc;
  for (int c = (int)a->nck - 1; c >= 0; --c) {
    BRT_CUDA_TRY(cudaStreamWaitEvent(rs, evRecomputed(c), 0));
    const AdjointState::Tape& tp = a->tape[c & 1];
    const uint32_t steps = std::min(a->k, a->T - (uint32_t)c * a->k);
    for (int s = (int)steps - 1; s >= 0; --s) {
      AdjointStepArgs R;
      std::memset(&R, 0, sizeof(R));
      R.posS = tp.pos + s * n; R.fwdS = tp.fwd + s * n; R.accS = tp.acc + s * n;
      R.lists = tp.lists + s * n * e->listStride; R.listStride = e->listStride;
      R.prev = tp.prev + s * n; R.idS = tp.id + s * n;
      R.flocks = e->flocks; R.agentBase = e->agentBase; R.obstacles = e->obstacles; R.obsMask = e->obsMask;
      R.nflocks = e->nflocks; R.n = e->N; R.dt = a->dt;
      R.gOutP = a->g[cur][0]; R.gOutF = a->g[cur][1]; R.gOutA = a->g[cur][2];
      R.gInP = a->g[cur ^ 1][0]; R.gInF = a->g[cur ^ 1][1]; R.gInA = a->g[cur ^ 1][2];
      R.contrib = a->contrib; R.selfP = a->selfP; R.selfF = a->selfF;
      R.inCount = a->inCount; R.inbox = a->inbox; R.inCap = a->inCap;
      R.ovHead = a->ovHead; R.ovNext = a->ovNext; R.entryStride = e->Mmax;
      R.accW = a->accW;
      if (e->adjointExport && a->expLists) {
        const size_t t = (size_t)c * a->k + s;
        R.exportLists = a->expLists + t * n * e->listStride;
        R.exportFlags = a->expFlags + t * n * 4;
        R.exportState = a->expState + t * n * 3;
      }
      BRT_CUDA_TRY(launchAdjointStep(R, rs));
      cur ^= 1;
    }
    BRT_CUDA_TRY(cudaEventRecord(evReversed(c), rs));
    if (c > 0 && (rc = recompute(c - 1))) return rc;
  }
  BRT_CUDA_TRY(cudaStreamWaitEvent(e->stream, evReversed(0), 0));
  FlockReduceArgs W;
  W.vals = a->accW; W.width = 3; W.agentBase = e->agentBase; W.nflocks = e->nflocks; W.out = a->gW;
  W.partial = a->partial;
  BRT_CUDA_TRY(launchFlockReduce(W, e->stream));
  OutArgs O;
  std::memset(&O, 0, sizeof(O));
  O.gP = a->g[cur][0]; O.gF = a->g[cur][1]; O.gA = a->g[cur][2];
  O.id0 = a->ckId; O.fwd0 = a->ckFwd; O.n = e->N;
  O.outP = a->io[0]; O.outF = a->io[1]; O.outA = a->io[2]; O.outV = a->io[3];
  BRT_CUDA_TRY(launchAdjointOut(O, e->stream));
  // Leave the engine at the forward's final state.
  if ((rc = copyState(e, e->posA, e->fwdA, e->accA, e->idA, a->finPos, a->finFwd, a->finAcc, a->finId))) return rc;
  if (e->Fs) BRT_CUDA_TRY(cudaMemcpyAsync(e->featA, a->finFeat, n * e->Fs * 4, cudaMemcpyDeviceToDevice, e->stream));
  return BRT_OK;
}

template <class Fn>
int runMaybeGraph(brt_engine* e, int kind, uint32_t variant, Fn enqueue) {
  AdjointState* a = e->adj;
  if (!e->adjointGraphs) return enqueue();
  uint32_t dtBits;
  std::memcpy(&dtBits, &a->dt, 4);
  auto key = std::make_tuple(kind, a->T, a->k, dtBits, e->paramsVersion, variant);
  auto it = a->graphs.find(key);
  if (it == a->graphs.end()) {
    if (a->graphs.size() >= 16) dropGraphs(a);
    cudaGraph_t g = nullptr;
    BRT_CUDA_TRY(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    e->capturing = true;
    int rc = enqueue();
    cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
    e->capturing = false;
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (ce != cudaSuccess) { setLastError(std::string("adjoint graph capture: ") + cudaGetErrorString(ce)); return BRT_ERR_CUDA; }
    cudaGraphExec_t ge = nullptr;
    ce = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) { setLastError(std::string("adjoint graph instantiate: ") + cudaGetErrorString(ce)); return BRT_ERR_CUDA; }
    it = a->graphs.emplace(key, ge).first;
  }
  BRT_CUDA_TRY(cudaGraphLaunch(it->second, e->stream));
  return BRT_OK;
}

cudaMemcpyKind kindIn(int where) { return where == BRT_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice; }
cudaMemcpyKind kindOut(int where) { return where == BRT_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice; }

__global__ void setWeightsKernel(FlockDev* flocks, const float* w, uint32_t nflocks) {
  const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nflocks) return;
  flocks[f].sep[0] = w[3 * f + 0];
  flocks[f].ali[0] = w[3 * f + 1];
  flocks[f].coh[0] = w[3 * f + 2];
}
__global__ void getWeightsKernel(const FlockDev* flocks, float* w, uint32_t nflocks) {
  const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nflocks) return;
  w[3 * f + 0] = flocks[f].sep[0];
  w[3 * f + 1] = flocks[f].ali[0];
  w[3 * f + 2] = flocks[f].coh[0];
}

}  // namespace
}  // namespace brt

using namespace brt;

extern "C" {

int brt_adjoint_forward(brt_engine* e, float elapsedTime, uint32_t nsteps, uint32_t checkpoint_every,
                        const float* target_pos4, int where, double* loss_per_flock) {
  brt::TraceRange trace(__func__);
  if (!e || !target_pos4 || nsteps == 0 || checkpoint_every == 0) { setLastError("brt_adjoint_forward: bad arguments"); return BRT_ERR_ARG; }
  if (where != BRT_MEM_HOST && where != BRT_MEM_DEVICE) return brt::argError(__func__);
  if (e->N == 0) return BRT_OK;
  int rc = checkSupported(e);
  if (rc) return rc;
  DeviceGuard guard(e->device);
  if (!e->adj) e->adj = new AdjointState();
  AdjointState* a = e->adj;
  const uint32_t k = std::min(checkpoint_every, nsteps);
  const uint32_t nck = (nsteps + k - 1) / k;
  if ((rc = ensureCapacity(e, nck, k, nsteps))) return rc;
  if (a->T != nsteps || a->k != k || a->dt != elapsedTime) dropGraphs(a);
  a->T = nsteps; a->k = k; a->nck = nck; a->dt = elapsedTime;
  a->taped = false;
  BRT_CUDA_TRY(cudaMemcpyAsync(a->target, target_pos4, (size_t)e->N * 16, kindIn(where), e->stream));
  if ((rc = runMaybeGraph(e, 0, 0u, [&] { return enqueueForward(e); }))) return rc;
  e->reordered = false;
  e->listsValid = false;
  if (loss_per_flock)
    BRT_CUDA_TRY(cudaMemcpyAsync(loss_per_flock, a->loss, 8 * (size_t)e->nflocks, kindOut(where), e->stream));
  a->taped = true;
  a->version = e->paramsVersion;
  a->weightsVersion = e->weightsVersion;
  if (where == BRT_MEM_HOST) return engineSyncAndCheck(e);
  return BRT_OK;
}

int brt_adjoint_backward(brt_engine* e, const double* loss_scale, const float* gpos4_T, const float* gfwd4_T,
                         const float* gacc4_T, int where_in, float* grad_pos4, float* grad_fwd4, float* grad_vel4,
                         float* grad_acc4, double* grad_weights, int where_out) {
  brt::TraceRange trace(__func__);
  if (!e) return brt::argError(__func__);
  if ((where_in != BRT_MEM_HOST && where_in != BRT_MEM_DEVICE) || (where_out != BRT_MEM_HOST && where_out != BRT_MEM_DEVICE))
    return brt::argError(__func__);
  AdjointState* a = e->adj;
  if (!a || !a->taped) { setLastError("brt_adjoint_backward: no taped forward (call brt_adjoint_forward first)"); return BRT_ERR_STATE; }
  if (a->version != e->paramsVersion || a->weightsVersion != e->weightsVersion) {
    setLastError("brt_adjoint_backward: parameters changed since the forward");
    return BRT_ERR_STATE;
  }
  if (e->adjointExport && a->capExport < a->T) { setLastError("brt_adjoint_backward: adjoint_export was enabled after the forward"); return BRT_ERR_STATE; }
  if (e->N == 0) return BRT_OK;
  DeviceGuard guard(e->device);
  const size_t n = e->N;
  uint32_t variant = 0;
  const float* extras[3] = {gpos4_T, gfwd4_T, gacc4_T};
  for (int c = 0; c < 3; ++c)
    if (extras[c]) {
      BRT_CUDA_TRY(cudaMemcpyAsync(a->io[c], extras[c], n * 16, kindIn(where_in), e->stream));
      variant |= 1u << c;
    }
  if (e->adjointExport) variant |= 16u;
  if (loss_scale) {
    std::vector<float> s(e->nflocks);
    for (uint32_t f = 0; f < e->nflocks; ++f) s[f] = (float)loss_scale[f];
    BRT_CUDA_TRY(cudaMemcpyAsync(a->scale, s.data(), 4 * s.size(), cudaMemcpyHostToDevice, e->stream));
    BRT_CUDA_TRY(cudaStreamSynchronize(e->stream));
    variant |= 8u;
  }
  int rc = runMaybeGraph(e, 1, variant, [&] { return enqueueBackward(e, variant); });
  if (rc) return rc;
  float* outs[4] = {grad_pos4, grad_fwd4, grad_acc4, grad_vel4};
  const int src[4] = {0, 1, 2, 3};
  for (int c = 0; c < 4; ++c)
    if (outs[c]) BRT_CUDA_TRY(cudaMemcpyAsync(outs[c], a->io[src[c]], n * 16, kindOut(where_out), e->stream));
  if (grad_weights)
    BRT_CUDA_TRY(cudaMemcpyAsync(grad_weights, a->gW, 24 * (size_t)e->nflocks, kindOut(where_out), e->stream));
  e->reordered = false;
  e->listsValid = false;
  if (where_out == BRT_MEM_HOST) return engineSyncAndCheck(e);
  return BRT_OK;
}

int brt_adjoint_get_tape(brt_engine* e, uint32_t* lists_by_id, uint32_t* flags_by_id, int where) {
  if (!e) return brt::argError(__func__);
  AdjointState* a = e->adj;
  if (!e->adjointExport || !a || !a->expLists || a->capExport < a->T) {
    setLastError("brt_adjoint_get_tape: enable option adjoint_export before brt_adjoint_forward");
    return BRT_ERR_STATE;
  }
  DeviceGuard guard(e->device);
  const size_t n = e->N;
  if (lists_by_id)
    BRT_CUDA_TRY(cudaMemcpyAsync(lists_by_id, a->expLists, n * a->T * e->listStride * 4, kindOut(where), e->stream));
  if (flags_by_id) BRT_CUDA_TRY(cudaMemcpyAsync(flags_by_id, a->expFlags, n * a->T * 16, kindOut(where), e->stream));
  if (where == BRT_MEM_HOST) return engineSyncAndCheck(e);
  return BRT_OK;
}

int brt_adjoint_get_tape_states(brt_engine* e, float* pos4, float* fwd4, float* acc4, int where) {
  if (!e) return brt::argError(__func__);
  AdjointState* a = e->adj;
  if (!e->adjointExport || !a || !a->expState || a->capExport < a->T) {
    setLastError("brt_adjoint_get_tape_states: enable option adjoint_export before brt_adjoint_forward");
    return BRT_ERR_STATE;
  }
  if (where != BRT_MEM_HOST && where != BRT_MEM_DEVICE) return brt::argError(__func__);
  DeviceGuard guard(e->device);
  const size_t n = e->N;
  float* dst[3] = {pos4, fwd4, acc4};
  for (int c = 0; c < 3; ++c) {
    if (!dst[c]) continue;
    // the tape holds (pos, fwd, acc) interleaved per agent; copy one of three
    BRT_CUDA_TRY(cudaMemcpy2DAsync(dst[c], 16, (const char*)a->expState + 16 * c, 48, 16, n * a->T, kindOut(where),
                                   e->stream));
  }
  if (where == BRT_MEM_HOST) return engineSyncAndCheck(e);
  return BRT_OK;
}

int brt_set_steering_weights(brt_engine* e, const float* weights3, int where) {
  if (!e || !weights3) return brt::argError(__func__);
  if (where != BRT_MEM_HOST && where != BRT_MEM_DEVICE) return brt::argError(__func__);
  DeviceGuard guard(e->device);
  e->weightsVersion++;
  if (where == BRT_MEM_HOST) {
    for (uint32_t f = 0; f < e->nflocks; ++f) {
      e->flocksHost[f].sep[0] = weights3[3 * f + 0];
      e->flocksHost[f].ali[0] = weights3[3 * f + 1];
      e->flocksHost[f].coh[0] = weights3[3 * f + 2];
      e->params[f].separationParams[0] = weights3[3 * f + 0];
      e->params[f].alignmentParams[0] = weights3[3 * f + 1];
      e->params[f].cohesionParams[0] = weights3[3 * f + 2];
    }
    BRT_CUDA_TRY(cudaMemcpyAsync(e->flocks, e->flocksHost.data(), sizeof(FlockDev) * e->nflocks, cudaMemcpyHostToDevice,
                                 e->stream));
    BRT_CUDA_TRY(cudaStreamSynchronize(e->stream));
  } else {
    setWeightsKernel<<<(e->nflocks + 127) / 128, 128, 0, e->stream>>>(e->flocks, weights3, e->nflocks);
    BRT_CUDA_TRY(cudaGetLastError());
    // The host copies follow on the next read back.
    std::vector<FlockDev> dev(e->nflocks);
    BRT_CUDA_TRY(cudaMemcpyAsync(dev.data(), e->flocks, sizeof(FlockDev) * e->nflocks, cudaMemcpyDeviceToHost, e->stream));
    BRT_CUDA_TRY(cudaStreamSynchronize(e->stream));
    for (uint32_t f = 0; f < e->nflocks; ++f) {
      e->flocksHost[f].sep[0] = dev[f].sep[0];
      e->flocksHost[f].ali[0] = dev[f].ali[0];
      e->flocksHost[f].coh[0] = dev[f].coh[0];
      e->params[f].separationParams[0] = dev[f].sep[0];
      e->params[f].alignmentParams[0] = dev[f].ali[0];
      e->params[f].cohesionParams[0] = dev[f].coh[0];
    }
  }
  return BRT_OK;
}

int brt_get_steering_weights(brt_engine* e, float* weights3, int where) {
  if (!e || !weights3) return brt::argError(__func__);
  if (where != BRT_MEM_HOST && where != BRT_MEM_DEVICE) return brt::argError(__func__);
  DeviceGuard guard(e->device);
  if (where == BRT_MEM_HOST) {
    for (uint32_t f = 0; f < e->nflocks; ++f) {
      weights3[3 * f + 0] = e->flocksHost[f].sep[0];
      weights3[3 * f + 1] = e->flocksHost[f].ali[0];
      weights3[3 * f + 2] = e->flocksHost[f].coh[0];
    }
    return BRT_OK;
  }
  getWeightsKernel<<<(e->nflocks + 127) / 128, 128, 0, e->stream>>>(e->flocks, weights3, e->nflocks);
  BRT_CUDA_TRY(cudaGetLastError());
  return BRT_OK;
}

}  // extern "C"
