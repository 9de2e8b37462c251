// brt_engine.cu -- host side of the C-ABI: engine lifetime, feature I/O,
// the fused step (optionally as one CUDA graph of many steps) and the
// stage-wise functionalities of the reference's plugin chain.
#include "brt_internal.cuh"
#include "brt_kernels.cuh"
#include "brt_engine_impl.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

namespace brt {

static thread_local std::string tlsLastError;
void setLastError(const std::string& msg) { tlsLastError = msg; }

// Largest float x with !(sqrtf(x) > r): the neighbour predicate
// !(sqrtf(d2) > r) of checkForNeighbor (Proximity3D_resources.cu:66-69) is
// then exactly d2 <= x, because sqrtf is monotone and correctly rounded on
// both host and device.
static float radiusThreshold(float r) {
  if (!(r >= 0.0f)) return -1.0f;
  if (std::isinf(r)) return INFINITY;
  float x = r * r;
  if (std::isinf(x)) x = 3.0e38f;
  while (!(std::sqrt(std::nextafter(x, INFINITY)) > r) && !std::isinf(std::nextafter(x, INFINITY))) x = std::nextafter(x, INFINITY);
  while (x > 0.0f && std::sqrt(x) > r) x = std::nextafter(x, 0.0f);
  return x;
}

// Smallest float x >= 0 with sqrtf(x) >= r, so that sqrtf(d2) < r is exactly
// d2 < x (0 when r <= 0: the test never holds).
static float lowerRadiusThreshold(float r) {
  if (!(r > 0.0f)) return 0.0f;
  if (std::isinf(r)) return INFINITY;
  float x = r * r;
  if (std::isinf(x)) return INFINITY;
  while (x > 0.0f && std::sqrt(std::nextafter(x, 0.0f)) >= r) x = std::nextafter(x, 0.0f);
  while (std::sqrt(x) < r) x = std::nextafter(x, INFINITY);
  return x;
}

static int validateParams(const brt_params& p, uint32_t& G) {
  if (p.disableSorting) { setLastError("disableSorting is not supported"); return BRT_ERR_CONFIG; }
  if (!(p.cellSize > 0.0f) || !(p.worldSize > 0.0f)) { setLastError("worldSize and cellSize must be positive"); return BRT_ERR_CONFIG; }
  double g = (double)p.worldSize / (double)p.cellSize;
  G = (uint32_t)std::llround(g);
  if (G < 3 || (float)G * p.cellSize != p.worldSize) {
    setLastError("worldSize must be gridSize * cellSize with gridSize >= 3");
    return BRT_ERR_CONFIG;
  }
  if ((double)G * G * G > (double)(1u << 30)) { setLastError("too many cells"); return BRT_ERR_CAPACITY; }
  if (p.maxNeighbors < 1 || p.maxNeighbors > BRT_MAX_NEIGHBORS) { setLastError("maxNeighbors must be in [1, 128]"); return BRT_ERR_CONFIG; }
  if (p.featuresCount > BRT_MAX_FEATUREDIM) { setLastError("featuresCount must be <= 32"); return BRT_ERR_CONFIG; }
  if (p.numObstacles > BRT_MAX_OBSTACLES) { setLastError("numObstacles must be <= 64"); return BRT_ERR_CONFIG; }
  if (!(p.commonMass != 0.0f)) { setLastError("commonMass must be nonzero"); return BRT_ERR_CONFIG; }
  if (p.schooling.mode < 0 || p.schooling.mode > 2) { setLastError("schooling.mode must be 0, 1 or 2"); return BRT_ERR_CONFIG; }
  if (p.schooling.mode != 0 && p.useKnn) { setLastError("schooling flocks use the first-M neighbour lists (useKnn = 0)"); return BRT_ERR_CONFIG; }
  return BRT_OK;
}

static FlockDev toDev(const brt_params& p, uint32_t G) {
  FlockDev d;
  std::memset(&d, 0, sizeof(d));
  d.G = G;
  d.C = G * G * G;
  d.n = p.numBodies;
  d.L = p.worldSize;
  d.cell = p.cellSize;
  {
    // exact reciprocal of a power-of-two cell (mantissa 0.5 after frexp),
    // when it is a normal float: x * invCell then equals x / cell bit for bit
    int ex = 0;
    const float m = std::frexp(p.cellSize, &ex);
    const float inv = std::ldexp(1.0f, 1 - ex);
    d.invCell = (m == 0.5f && std::isnormal(inv) && inv * p.cellSize == 1.0f) ? inv : 0.0f;
  }
  d.radius = p.commonSearchRadius;
  d.r2thr = radiusThreshold(p.commonSearchRadius);
  d.M = p.maxNeighbors;
  d.maxPerCell = p.maxBodiesPerCell;
  d.useKnn = p.useKnn;
  d.maxSpeed = p.commonMaxSpeed;
  d.maxForce = p.commonMaxForce;
  d.mass = p.commonMass;
  d.minR = p.commonSensingMinRadius;
  for (int k = 0; k < 3; ++k) { d.sep[k] = p.separationParams[k]; d.ali[k] = p.alignmentParams[k]; d.coh[k] = p.cohesionParams[k]; }
  d.use2D = p.use2DProjection;
  d.F = p.featuresCount;
  d.relax = p.featureRelaxRate;
  d.clus = p.clusteringForceParams[0];
  d.aclus = p.alignmentClusteringForceParams[0];
  for (int k = 0; k < 3; ++k) d.simStats[k] = p.similarityStatsParams[k];
  d.avgCtl = p.avgSimilarityController;
  d.numObstacles = p.numObstacles;
  d.obsW = p.obstacleAvoidanceWeight;
  d.minT = lowerRadiusThreshold(p.commonSensingMinRadius);
  d.sepT = radiusThreshold(p.separationParams[1]);
  d.aliT = radiusThreshold(p.alignmentParams[1]);
  d.cohT = radiusThreshold(p.cohesionParams[1]);
  {
    const float mc = std::max(p.separationParams[2], std::max(p.alignmentParams[2], p.cohesionParams[2]));
    d.cosBound2 = (mc < -1.0f) ? mc * mc : 0.0f;
  }
  d.school = p.schooling.mode;
  d.schTheta = p.schooling.theta;
  d.schRr = p.schooling.r_r;
  d.schRp = p.schooling.r_p;
  d.schEta = p.schooling.eta;
  d.schWa = p.schooling.w_a;
  d.schWo = p.schooling.w_o;
  d.schS = p.schooling.s;
  d.schRand = p.schooling.randomDeviationWeight;
  d.schSeed = p.schooling.seed;
  return d;
}

// Distance on a circle of circumference L from c to the arc [a, b].
static double arcGap(double c, double a, double b, double L) {
  double t = std::fmod(c - a, L);
  if (t < 0) t += L;
  if (t <= b - a) return 0.0;
  auto circ = [L](double x) { x = std::fmod(std::fabs(x), L); return std::min(x, L - x); };
  return std::min(circ(c - a), circ(c - b));
}

// The obstacle field of one flock on its EnvGrid3D grid: bit o of a cell's
// mask is set when obstacle o's reach (radius + commonSearchRadius, as the
// kernels compute it in float) comes within a small margin of the cell's box
// under the periodic wrap, so the set is a superset of the obstacles that
// any position in the cell can feel.  Entries are at the flock's global
// cell indices.
static void buildObstacleField(const brt_params& p, const FlockDev& d, std::vector<uint2>& mask) {
  const double L = d.L, cell = d.cell;
  for (uint32_t c = 0; c < d.C; ++c) mask[d.cellBase + c] = make_uint2(0u, 0u);
  std::vector<double> gap[3];
  for (uint32_t o = 0; o < p.numObstacles; ++o) {
    const float reachF = p.obstacles[o][3] + p.commonSearchRadius;
    const double reach = (double)reachF + 1e-3 + 1e-5 * L;
    for (int ax = 0; ax < 3; ++ax) {
      gap[ax].assign(d.G, 0.0);
      for (uint32_t g = 0; g < d.G; ++g) gap[ax][g] = arcGap(p.obstacles[o][ax], g * cell, (g + 1) * cell, L);
    }
    for (uint32_t gz = 0; gz < d.G; ++gz) {
      if (gap[2][gz] > reach) continue;
      for (uint32_t gy = 0; gy < d.G; ++gy) {
        if (gap[1][gy] > reach) continue;
        for (uint32_t gx = 0; gx < d.G; ++gx) {
          const double q = gap[0][gx] * gap[0][gx] + gap[1][gy] * gap[1][gy] + gap[2][gz] * gap[2][gz];
          if (gap[0][gx] > reach || q > reach * reach) continue;
          uint2& m = mask[d.cellBase + (gz * d.G + gy) * d.G + gx];
          if (o < 32) m.x |= 1u << o; else m.y |= 1u << (o - 32);
        }
      }
    }
  }
}

}  // namespace brt

using namespace brt;


namespace {

__global__ void iotaKernel(uint32_t* a, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = i;
}
cudaError_t launchIota(uint32_t* a, uint32_t n, cudaStream_t st) {
  iotaKernel<<<(n + 255) / 256, 256, 0, st>>>(a, n);
  return cudaGetLastError();
}

// The re-sort's state as after creation: no previous order, empty mover
// lists (kNoMover heads), zero counters and look-back words.
cudaError_t resetResort(brt_engine* e) {
  cudaError_t err = cudaMemsetAsync(e->resortMem, 0, e->resortWords * 4, e->stream);
  if (err == cudaSuccess && e->C) err = cudaMemsetAsync(e->rsHead, 0xFF, (size_t)e->C * 4, e->stream);
  return err;
}

void freeAll(brt_engine* e) {
  freeAdjoint(e->adj);
  e->adj = nullptr;
  for (auto& kv : e->graphs) cudaGraphExecDestroy(kv.second);
  e->graphs.clear();
  for (int r = 0; r < brt_engine::kRing; ++r)
    for (int k = 0; k < 5; ++k)
      if (e->ev[r][k]) cudaEventDestroy(e->ev[r][k]);
  void* ptrs[] = {e->flocks, e->agentBase, e->obstacles, e->obsMask, e->posA, e->fwdA, e->accA, e->posS, e->fwdS, e->accS,
                  e->featA, e->featS, e->idA, e->idS, e->statsById, e->steer, e->lists, e->pairs[0], e->pairs[1],
                  e->cellStart, e->cellEnd, e->sortMem, e->errWord, e->stage4, e->stageF, e->stepCounter, e->cullWords,
                  e->membership[0], e->membership[1], e->resortMem};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (e->tiles) cudaFree(e->tiles);
  if (e->tileCounter) cudaFree(e->tileCounter);
  for (auto& u : e->user) {
    cudaFree(u.a);
    cudaFree(u.s);
  }
  e->user.clear();
  if (e->userIds.a) cudaFree(e->userIds.a);
  if (e->userIds.s) cudaFree(e->userIds.s);
  if (e->userStage) cudaFree(e->userStage);
  if (e->stream) cudaStreamDestroy(e->stream);
}

HashArgs hashArgs(brt_engine* e) {
  HashArgs A;
  std::memset(&A, 0, sizeof(A));
  A.pos = e->posA; A.id = e->idA; A.pairs = e->pairs[0];
  A.flocks = e->flocks; A.agentBase = e->agentBase; A.nflocks = e->nflocks; A.n = e->N;
  A.passes = e->plan.passes; A.bins = e->plan.bins;
  for (uint32_t k = 0; k < e->plan.passes; ++k) { A.shift[k] = e->plan.shift[k]; A.mask[k] = sortPassMask(e->plan, k); }
  A.hist = e->ss.hist;
  A.cellStart = e->cellStart; A.cellEnd = e->cellEnd; A.cellWords4 = e->Cpad / 4;
  A.status = e->ss.status; A.statusWords = e->plan.passes * std::max(1u, e->plan.tiles) * e->plan.bins;
  A.counters = e->ss.counters;
  A.stepCounter = e->stepCounter;
  return A;
}

StageArgs stageArgs(brt_engine* e) {
  StageArgs A;
  std::memset(&A, 0, sizeof(A));
  A.posS = e->posS; A.fwdS = e->fwdS; A.accS = e->accS; A.featS = e->featS; A.idS = e->idS;
  A.posA = e->posA; A.fwdA = e->fwdA; A.accA = e->accA; A.featA = e->featA; A.idA = e->idA;
  A.statsById = e->statsById; A.steer = e->steer; A.fwdW = e->fwdS;
  A.cellStart = e->cellStart; A.cellEnd = e->cellEnd;
  A.flocks = e->flocks; A.agentBase = e->agentBase; A.obstacles = e->obstacles; A.obsMask = e->obsMask;
  A.lists = e->lists; A.listStride = e->listStride;
  A.nflocks = e->nflocks; A.n = e->N; A.Fs = e->Fs;
  A.stepCounter = e->stepCounter;
  return A;
}

// Drains one ring slot of stage events into the totals.
int drainSlot(brt_engine* e, int r) {
  if (!e->pending[r]) return BRT_OK;
  BRT_CUDA_TRY(cudaEventSynchronize(e->ev[r][4]));
  for (int k = 0; k < 4; ++k) {
    float ms = 0.0f;
    BRT_CUDA_TRY(cudaEventElapsedTime(&ms, e->ev[r][k], e->ev[r][k + 1]));
    e->stageMs[k] += ms;
  }
  e->timedSteps++;
  e->pending[r] = false;
  return BRT_OK;
}

// Records stage boundary k of the current timed step.
int stageMark(brt_engine* e, int k) {
  if (!e->timing || e->capturing) return BRT_OK;
  BRT_CUDA_TRY(cudaEventRecord(e->ev[e->ringPos][k], e->stream));
  return BRT_OK;
}

// hash -> sort -> reorder + cell ranges
ResortArgs resortArgs(brt_engine* e) {
  ResortArgs A{};
  A.pos = e->posA; A.id = e->idA; A.prevPairs = e->pairs[e->plan.passes & 1];
  A.cellStart = e->cellStart; A.cellEnd = e->cellEnd;
  A.flocks = e->flocks; A.agentBase = e->agentBase;
  A.nflocks = e->nflocks; A.n = e->N; A.numCells = e->C;
  A.maxMovers = e->N / 8;
  A.newKey = e->rsNewKey; A.prefix = e->rsPrefix; A.blockStay = e->rsBlockStay;
  A.moverCount = e->rsCount; A.moverHead = e->rsHead; A.moverNext = e->rsNext;
  A.newStart = e->rsNewStart; A.stayBase = e->rsStayBase; A.tileStatus = e->rsTiles; A.tileCounter = e->rsCounter; A.words = e->rsWords;
  A.stepCounter = e->stepCounter;
  A.out = e->pairs[e->plan.passes & 1];
  A.errWord = e->errWord;
  A.wait = e->wait;
  return A;
}

// The next fused step cannot take its order from the current one (the
// canonical arrays or the sort plan were replaced): it runs the full sort.
cudaError_t invalidateResort(brt_engine* e) {
  return cudaMemsetAsync(e->rsWords + kResortWordValid, 0, 4, e->stream);
}

// Hash, sort and reorder.  From the fused step (incremental) the order comes
// from the incremental re-sort when the previous step's order allows it, the
// hash and radix passes running only otherwise (decided on the device).
int enqueueReorder(brt_engine* e, bool incremental = false) {
  cudaStream_t st = e->stream;
  int rc = stageMark(e, 0);
  if (rc) return rc;
  const bool rs = incremental && e->resortOn;
  HashArgs H = hashArgs(e);
  H.resortValid = e->rsWords + kResortWordValid;
  const uint32_t* gate = nullptr;
  ResortArgs RS;
  if (rs) {
    RS = resortArgs(e);
    BRT_CUDA_TRY(launchResortMark(RS, st));
    gate = e->rsWords + kResortWordMode;
    H.gate = gate;
  }
  BRT_CUDA_TRY(launchHash(H, e->smCount * 8, st));
  if ((rc = stageMark(e, 1))) return rc;
  for (uint32_t k = 0; k < e->plan.passes; ++k)
    BRT_CUDA_TRY(launchOnesweepPass(e->plan, k, e->pairs[k & 1], e->pairs[(k + 1) & 1], e->ss, e->errWord, st, gate));
  if (rs) BRT_CUDA_TRY(launchResortPlace(RS, st));
  if ((rc = stageMark(e, 2))) return rc;
  e->finalPairs = e->plan.passes & 1;
  ReorderArgs R;
  std::memset(&R, 0, sizeof(R));
  R.pairs = e->pairs[e->finalPairs];
  R.posA = e->posA; R.fwdA = e->fwdA; R.accA = e->accA; R.featA = e->featA; R.idA = e->idA;
  R.posS = e->posS; R.fwdS = e->fwdS; R.accS = e->accS; R.featS = e->featS; R.idS = e->idS;
  R.prevOut = e->tapePrev;
  R.fs4 = e->Fs / 4;
  R.cellStart = e->cellStart; R.cellEnd = e->cellEnd;
  R.hist = e->ss.hist; R.histWords = e->plan.passes * e->plan.bins;
  R.n = e->N; R.numCells = e->C; R.errWord = e->errWord;
  if (e->scanVariant == 0 || e->scanVariant == 1) {
    R.cullWords = e->cullWords;
    R.flocks = e->flocks; R.agentBase = e->agentBase; R.nflocks = e->nflocks;
  }
  if (rs) {
    R.resortMode = e->rsWords + kResortWordMode;
    R.newStart = e->rsNewStart;
    R.moverCount = e->rsCount; R.moverHead = e->rsHead;
    R.resortValid = e->rsWords + kResortWordValid;
  }
  BRT_CUDA_TRY(launchReorder(R, st));
  // registered arrays move with their agents (slot i takes the previous slot
  // pairs[i].y), the agent-id map with them
  if (!e->user.empty() && !e->userFrozen) {
    const uint32_t* prev = reinterpret_cast<const uint32_t*>(e->pairs[e->finalPairs]) + 1;
    auto permute = [&](brt_engine::UserArray& u) -> cudaError_t {
      cudaError_t err = launchGatherWords(u.a, prev, 2, u.s, u.words, e->N, st);
      if (err != cudaSuccess) return err;
      return cudaMemcpyAsync(u.a, u.s, (size_t)e->N * u.words * 4, cudaMemcpyDeviceToDevice, st);
    };
    BRT_CUDA_TRY(permute(e->userIds));
    for (auto& u : e->user) BRT_CUDA_TRY(permute(u));
  }
  return stageMark(e, 3);
}

int enqueueStep(brt_engine* e, float dt, bool record) {
  const bool timed = e->timing && !e->capturing;
  if (timed) {
    int rc = drainSlot(e, e->ringPos);
    if (rc) return rc;
  }
  int rc = enqueueReorder(e, true);
  if (rc) return rc;
  FusedArgs F;
  std::memset(&F, 0, sizeof(F));
  F.posS = e->posS; F.fwdS = e->fwdS; F.accS = e->accS; F.featS = e->featS; F.idS = e->idS;
  F.posA = e->posA; F.fwdA = e->fwdA; F.accA = e->accA; F.featA = e->featA; F.idA = e->idA;
  F.statsById = e->statsById;
  F.cellStart = e->cellStart; F.cellEnd = e->cellEnd;
  F.flocks = e->flocks; F.agentBase = e->agentBase; F.obstacles = e->obstacles; F.obsMask = e->obsMask;
  F.lists = record ? e->lists : nullptr; F.listStride = e->listStride;
  F.nflocks = e->nflocks; F.n = e->N; F.Mmax = e->Mmax; F.Fs = e->Fs; F.dt = dt;
  F.scanVariant = e->scanVariant;
  F.tiles = e->tiles; F.numTiles = e->numTiles; F.tileCounter = e->tileCounter; F.tileBlocks = e->tileBlocks;
  F.stepCounter = e->stepCounter;
  F.cullGate = (e->scanVariant == 0 || e->scanVariant == 1) ? e->cullWords + 2 : nullptr;
  // The single-pass kernel covers every flock unless one needs clustering
  // steering (it needs the whole list first) or kNN lists longer than a warp.
  // kNN flocks take its cooperative kNN scan (scan 8).
  bool twoPass = e->forceTwoPass || (e->anyKnn && e->Mmax > 32);
  for (const FlockDev& d : e->flocksHost) twoPass = twoPass || (d.F > 0 && (d.clus != 0.0f || d.aclus != 0.0f));
  if (e->anyKnn && !twoPass) F.scanVariant = 8;
  if (e->school) BRT_CUDA_TRY(launchSchool(F, e->stream));
  else if (twoPass) BRT_CUDA_TRY(launchFused(F, e->anyKnn, e->stream));
  else BRT_CUDA_TRY(launchFlock(F, e->phase2Variant, e->fusedBlock, e->regBudget, e->stream));
  if (timed) {
    if ((rc = stageMark(e, 4))) return rc;
    e->pending[e->ringPos] = true;
    e->ringPos = (e->ringPos + 1) % brt_engine::kRing;
  }
  return BRT_OK;
}

// Captures the nsteps-step graph (cached by dt, nsteps, recording, params).
int getGraph(brt_engine* e, float dt, uint32_t nsteps, bool record, cudaGraphExec_t* out) {
  uint32_t dtBits;
  std::memcpy(&dtBits, &dt, 4);
  auto key = std::make_tuple(nsteps, dtBits, record, e->paramsVersion);
  auto it = e->graphs.find(key);
  if (it == e->graphs.end()) {
    if (e->graphs.size() >= 8) {
      for (auto& kv : e->graphs) cudaGraphExecDestroy(kv.second);
      e->graphs.clear();
    }
    cudaGraph_t g = nullptr;
    BRT_CUDA_TRY(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    e->capturing = true;
    int rc = BRT_OK;
    for (uint32_t s = 0; s < nsteps && !rc; ++s) rc = enqueueStep(e, dt, record);
    cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
    e->capturing = false;
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (ce != cudaSuccess) { setLastError(std::string("graph capture: ") + cudaGetErrorString(ce)); return BRT_ERR_CUDA; }
    cudaGraphExec_t ge = nullptr;
    ce = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) { setLastError(std::string("graph instantiate: ") + cudaGetErrorString(ce)); return BRT_ERR_CUDA; }
    it = e->graphs.emplace(key, ge).first;
  }
  *out = it->second;
  return BRT_OK;
}

int checkDeviceError(brt_engine* e, bool clear) {
  uint32_t w = 0;
  BRT_CUDA_TRY(cudaMemcpyAsync(&w, e->errWord, 4, cudaMemcpyDeviceToHost, e->stream));
  BRT_CUDA_TRY(cudaStreamSynchronize(e->stream));
  if (w) e->stateLost = true;
  if (w && clear) BRT_CUDA_TRY(cudaMemsetAsync(e->errWord, 0, 4, e->stream));
  if (w & kDevErrLookback) { setLastError("onesweep look-back spin limit reached"); return BRT_ERR_TIMEOUT; }
  if (w) { setLastError("device-side pipeline check failed"); return BRT_ERR_STATE; }
  return BRT_OK;
}

int syncAndCheck(brt_engine* e) { return checkDeviceError(e, true); }

int configureKernels(brt_engine* e);

// The (flock, row segment) tiles of scan variant 6: every x-row of every
// flock cut into segments of at most kTileMaxCells home cells.
int buildTiles(brt_engine* e) {
  std::vector<uint4> tiles;
  for (uint32_t f = 0; f < e->nflocks; ++f) {
    const FlockDev& d = e->flocksHost[f];
    const uint32_t G = d.G;
    const uint32_t R = std::min<uint32_t>(G, kTileMaxCells);
    for (uint32_t z = 0; z < G; ++z)
      for (uint32_t y = 0; y < G; ++y)
        for (uint32_t x0 = 0; x0 < G; x0 += R)
          tiles.push_back(make_uint4(f, y | (z << 16), x0 | (std::min(R, G - x0) << 16), 0u));
  }
  e->numTiles = (uint32_t)tiles.size();
  if (tiles.empty()) return BRT_OK;
  BRT_CUDA_TRY(cudaMalloc(&e->tiles, tiles.size() * sizeof(uint4)));
  BRT_CUDA_TRY(cudaMalloc(&e->tileCounter, 4));
  BRT_CUDA_TRY(cudaMemcpy(e->tiles, tiles.data(), tiles.size() * sizeof(uint4), cudaMemcpyHostToDevice));
  e->tileBlocks = std::min<uint32_t>(e->numTiles, tileFlockBlocks(e->Mmax, e->Fs, (int)e->smCount));
  return BRT_OK;
}

}  // namespace

namespace brt {
int engineEnqueueStep(brt_engine* e, float dt, bool record) { return enqueueStep(e, dt, record); }
cudaError_t engineInvalidateResort(brt_engine* e) { return invalidateResort(e); }
int engineSyncAndCheck(brt_engine* e) { return syncAndCheck(e); }
}  // namespace brt

// ---------------------------------------------------------------------------
extern "C" {

const char* brt_version(void) { return "behavert_b200 0.1 (sm_100a)"; }

const char* brt_error_string(int status) {
  switch (status) {
    case BRT_OK: return "ok";
    case BRT_ERR_CUDA: return "CUDA error";
    case BRT_ERR_CONFIG: return "invalid configuration";
    case BRT_ERR_CAPACITY: return "capacity exceeded";
    case BRT_ERR_TIMEOUT: return "device wait timed out";
    case BRT_ERR_ARG: return "invalid argument";
    case BRT_ERR_STATE: return "invalid call order";
    case BRT_ERR_NODEVICE: return "no CUDA device";
    default: return "unknown status";
  }
}

const char* brt_last_error(void) { return tlsLastError.c_str(); }

int brt_device_count(int* count) {
  if (!count) return brt::argError(__func__);
  *count = 0;
  cudaError_t err = cudaGetDeviceCount(count);
  if (err != cudaSuccess) { *count = 0; cudaGetLastError(); }
  return BRT_OK;
}

int brt_params_default(brt_params* p) {
  if (!p) return brt::argError(__func__);
  std::memset(p, 0, sizeof(*p));
  p->numBodies = 4096;
  p->commonRadius = 1.0f;
  p->worldSize = 64.0f;
  p->cellSize = 4.0f;
  p->maxBodiesPerCell = 0;
  p->maxNeighbors = 16;
  p->useKnn = 0;
  p->commonSearchRadius = 4.0f;
  p->commonMaxSpeed = 1.0f;
  p->commonMaxForce = 0.1f;
  p->commonMass = 1.0f;
  p->commonSensingMinRadius = 0.0f;
  p->separationParams[0] = 1.5f; p->separationParams[1] = 4.0f; p->separationParams[2] = -2.0f;
  p->alignmentParams[0] = 1.0f; p->alignmentParams[1] = 4.0f; p->alignmentParams[2] = -2.0f;
  p->cohesionParams[0] = 1.0f; p->cohesionParams[1] = 4.0f; p->cohesionParams[2] = -2.0f;
  p->featuresCount = 0;
  p->similarityStatsParams[0] = 0.01f; p->similarityStatsParams[1] = 0.1f; p->similarityStatsParams[2] = 0.001f;
  p->avgSimilarityController = 1.0f;
  p->featureRelaxRate = 0.0f;
  // SchoolingPlugIn::install (PlugIns/Schooling/include/SchoolingPlugIn.h:115-160)
  p->schooling.mode = 0;
  p->schooling.theta = (float)std::cos(0.1);
  p->schooling.delta = 0.01f;
  p->schooling.r_r = 1.0f;
  p->schooling.r_p = p->commonSearchRadius;
  p->schooling.eta = (float)std::cos(3.05);
  p->schooling.w_a = 1.0f;
  p->schooling.w_o = 16.0f;
  p->schooling.s = 3.0f;
  p->schooling.randomDeviationWeight = 0.1f;
  p->schooling.seed = 0;
  return BRT_OK;
}

int brt_engine_create(const brt_params* flocks, uint32_t num_flocks, int device, brt_engine** out) {
  brt::TraceRange trace(__func__);
  if (!flocks || !out || num_flocks == 0) { setLastError("brt_engine_create: bad arguments"); return BRT_ERR_ARG; }
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); setLastError("no CUDA device"); return BRT_ERR_NODEVICE; }
  if (device < 0 || device >= ndev) { setLastError("bad device index"); return BRT_ERR_ARG; }
  DeviceGuard guard(device);
  brt_engine* e = new brt_engine();
  e->device = device;
  e->nflocks = num_flocks;
  e->params.assign(flocks, flocks + num_flocks);
  std::vector<uint32_t> agentBase(num_flocks + 1, 0);
  std::vector<float4> obs;
  uint64_t N = 0, C = 0;
  for (uint32_t f = 0; f < num_flocks; ++f) {
    uint32_t G = 0;
    int rc = validateParams(flocks[f], G);
    if (rc) { delete e; return rc; }
    FlockDev d = toDev(flocks[f], G);
    d.cellBase = (uint32_t)C;
    d.agentBase = (uint32_t)N;
    d.obsBase = (uint32_t)obs.size();
    for (uint32_t o = 0; o < flocks[f].numObstacles; ++o)
      obs.push_back(make_float4(flocks[f].obstacles[o][0], flocks[f].obstacles[o][1], flocks[f].obstacles[o][2], flocks[f].obstacles[o][3]));
    agentBase[f] = (uint32_t)N;
    N += flocks[f].numBodies;
    C += d.C;
    e->Mmax = std::max(e->Mmax, d.M);
    e->Fmax = std::max(e->Fmax, d.F);
    e->anyKnn = e->anyKnn || d.useKnn;
    if (f > 0 && (d.school != 0) != e->school) {
      delete e;
      setLastError("all flocks of an engine use the same steering family (schooling.mode 0, or 1/2)");
      return BRT_ERR_CONFIG;
    }
    e->school = d.school != 0;
    e->flocksHost.push_back(d);
  }
  // Neighbour-list entries hold a 26-bit sorted slot (brt_fused.cu).
  if (N >= (1ull << 26) || C >= (1ull << 30)) {
    delete e;
    setLastError("too many agents (at most 2^26 - 1) or cells (at most 2^30 - 1) in one engine");
    return BRT_ERR_CAPACITY;
  }
  agentBase[num_flocks] = (uint32_t)N;
  e->N = (uint32_t)N;
  e->C = (uint32_t)C;
  e->Cpad = (e->C + 3) & ~3u;
  e->Fs = (e->Fmax + 3) & ~3u;
  e->listStride = e->Mmax + 1;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) e->smCount = prop.multiProcessorCount;
  uint32_t bits = 1;
  while ((1ull << bits) < C) ++bits;
  e->plan = makeSortPlan(e->N, bits, 8);
  int rc = BRT_OK;
  auto chk = [&](int r) { if (r && !rc) rc = r; };
  if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) { delete e; setLastError("stream creation failed"); return BRT_ERR_CUDA; }
  const size_t n = e->N;
  chk(devAlloc(&e->flocks, num_flocks));
  chk(devAlloc(&e->agentBase, num_flocks + 1));
  chk(devAlloc(&e->obstacles, std::max<size_t>(1, obs.size())));
  if (!obs.empty()) chk(devAlloc(&e->obsMask, e->C));
  chk(devAlloc(&e->posA, n)); chk(devAlloc(&e->fwdA, n)); chk(devAlloc(&e->accA, n));
  chk(devAlloc(&e->posS, n)); chk(devAlloc(&e->fwdS, n)); chk(devAlloc(&e->accS, n));
  chk(devAlloc(&e->featA, n * e->Fs)); chk(devAlloc(&e->featS, n * e->Fs));
  chk(devAlloc(&e->idA, n)); chk(devAlloc(&e->idS, n));
  chk(devAlloc(&e->statsById, n));
  chk(devAlloc(&e->steer, n));
  chk(devAlloc(&e->lists, n * e->listStride));
  chk(devAlloc(&e->pairs[0], n)); chk(devAlloc(&e->pairs[1], n));
  chk(devAlloc(&e->cellStart, e->Cpad)); chk(devAlloc(&e->cellEnd, e->Cpad));
  chk(devAlloc(&e->errWord, 1));
  chk(devAlloc(&e->stepCounter, 1));
  chk(devAlloc(&e->cullWords, 4));
  chk(devAlloc(&e->stage4, n));
  chk(devAlloc(&e->stageF, std::max<size_t>(1, n * e->Fmax)));
  const size_t sortBytes = sortScratchBytes(e->plan, false);
  if (!rc && cudaMalloc(&e->sortMem, sortBytes) != cudaSuccess) { setLastError("sort scratch allocation failed"); rc = BRT_ERR_CUDA; }
  // incremental re-sort arrays, each on a 16-byte boundary
  auto words4 = [](size_t w) { return (w + 3) & ~(size_t)3; };
  const size_t rsSizes[11] = {n, n, n, (size_t)resortBlocks(e->N) + 1, e->C, e->C, e->C,
                              std::max<size_t>(1, resortCellTiles(e->C)), 1, kResortWords, e->C};
  size_t rsWordsTotal = 0;
  for (size_t w : rsSizes) rsWordsTotal += words4(w);
  if (!rc && cudaMalloc(&e->resortMem, rsWordsTotal * 4) != cudaSuccess) { setLastError("re-sort allocation failed"); rc = BRT_ERR_CUDA; }
  e->resortWords = rsWordsTotal;
  if (rc) { freeAll(e); delete e; return rc; }
  {
    uint32_t** rsPtrs[11] = {&e->rsNewKey, &e->rsPrefix, &e->rsNext, &e->rsBlockStay, &e->rsCount, &e->rsHead,
                             &e->rsNewStart, &e->rsTiles, &e->rsCounter, &e->rsWords, &e->rsStayBase};
    size_t off = 0;
    for (int k = 0; k < 11; ++k) { *rsPtrs[k] = e->resortMem + off; off += words4(rsSizes[k]); }
  }
  e->ss = carveSortScratch(e->plan, e->sortMem, false);
  cudaStream_t st = e->stream;
  BRT_CUDA_TRY(cudaMemcpyAsync(e->flocks, e->flocksHost.data(), sizeof(FlockDev) * num_flocks, cudaMemcpyHostToDevice, st));
  BRT_CUDA_TRY(cudaMemcpyAsync(e->agentBase, agentBase.data(), 4 * (num_flocks + 1), cudaMemcpyHostToDevice, st));
  if (!obs.empty()) {
    BRT_CUDA_TRY(cudaMemcpyAsync(e->obstacles, obs.data(), sizeof(float4) * obs.size(), cudaMemcpyHostToDevice, st));
    std::vector<uint2> field(e->C, make_uint2(0u, 0u));
    for (uint32_t f = 0; f < num_flocks; ++f) buildObstacleField(flocks[f], e->flocksHost[f], field);
    BRT_CUDA_TRY(cudaMemcpyAsync(e->obsMask, field.data(), sizeof(uint2) * field.size(), cudaMemcpyHostToDevice, st));
    BRT_CUDA_TRY(cudaStreamSynchronize(st));
  }
  BRT_CUDA_TRY(cudaMemsetAsync(e->sortMem, 0, sortBytes, st));
  BRT_CUDA_TRY(resetResort(e));
  if (n) {
    BRT_CUDA_TRY(cudaMemsetAsync(e->pairs[0], 0, n * 8, st));
    BRT_CUDA_TRY(cudaMemsetAsync(e->pairs[1], 0, n * 8, st));
  }
  BRT_CUDA_TRY(cudaMemsetAsync(e->errWord, 0, 4, st));
  BRT_CUDA_TRY(cudaMemsetAsync(e->stepCounter, 0, 4, st));
  BRT_CUDA_TRY(cudaMemsetAsync(e->cullWords, 0, 16, st));
  if (n) {
    BRT_CUDA_TRY(cudaMemsetAsync(e->posA, 0, n * 16, st));
    BRT_CUDA_TRY(cudaMemsetAsync(e->fwdA, 0, n * 16, st));
    BRT_CUDA_TRY(cudaMemsetAsync(e->accA, 0, n * 16, st));
    BRT_CUDA_TRY(cudaMemsetAsync(e->statsById, 0, n * 16, st));
    BRT_CUDA_TRY(cudaMemsetAsync(e->steer, 0, n * 16, st));
    if (e->Fs) BRT_CUDA_TRY(cudaMemsetAsync(e->featA, 0, n * e->Fs * 4, st));
    // identity slot order
    std::vector<uint32_t> iota(n);
    for (size_t i = 0; i < n; ++i) iota[i] = (uint32_t)i;
    BRT_CUDA_TRY(cudaMemcpyAsync(e->idA, iota.data(), 4 * n, cudaMemcpyHostToDevice, st));
    BRT_CUDA_TRY(cudaStreamSynchronize(st));
  }
  rc = configureKernels(e);
  if (rc) { freeAll(e); delete e; return rc; }
  rc = buildTiles(e);
  if (rc) { freeAll(e); delete e; return rc; }
  BRT_CUDA_TRY(cudaStreamSynchronize(st));
  *out = e;
  return BRT_OK;
}

int brt_engine_destroy(brt_engine* e) {
  brt::TraceRange trace(__func__);
  if (!e) return brt::argError(__func__);
  DeviceGuard guard(e->device);
  cudaStreamSynchronize(e->stream);
  freeAll(e);
  delete e;
  return BRT_OK;
}

int brt_engine_num_agents(const brt_engine* e, uint32_t* n) {
  if (!e || !n) return brt::argError(__func__);
  *n = e->N;
  return BRT_OK;
}
int brt_engine_num_cells(const brt_engine* e, uint32_t* c) {
  if (!e || !c) return brt::argError(__func__);
  *c = e->C;
  return BRT_OK;
}
int brt_neighbor_list_stride(const brt_engine* e, uint32_t* stride) {
  if (!e || !stride) return brt::argError(__func__);
  *stride = e->listStride;
  return BRT_OK;
}

int brt_engine_set_params(brt_engine* e, uint32_t flock, const brt_params* p) {
  if (!e || !p || flock >= e->nflocks) { setLastError("brt_engine_set_params: bad arguments"); return BRT_ERR_ARG; }
  const brt_params& o = e->params[flock];
  if (p->numBodies != o.numBodies || p->worldSize != o.worldSize || p->cellSize != o.cellSize ||
      p->maxNeighbors != o.maxNeighbors || p->featuresCount != o.featuresCount || p->numObstacles != o.numObstacles ||
      (p->useKnn != 0) != (o.useKnn != 0) || (p->schooling.mode != 0) != (o.schooling.mode != 0)) {
    setLastError("brt_engine_set_params: geometry fields cannot change");
    return BRT_ERR_CONFIG;
  }
  uint32_t G = 0;
  int rc = validateParams(*p, G);
  if (rc) return rc;
  DeviceGuard guard(e->device);
  FlockDev d = toDev(*p, G);
  const FlockDev& old = e->flocksHost[flock];
  d.cellBase = old.cellBase;
  d.agentBase = old.agentBase;
  d.obsBase = old.obsBase;
  e->flocksHost[flock] = d;
  e->params[flock] = *p;
  BRT_CUDA_TRY(cudaMemcpyAsync(e->flocks + flock, &e->flocksHost[flock], sizeof(FlockDev), cudaMemcpyHostToDevice, e->stream));
  std::vector<float4> obs;
  for (uint32_t k = 0; k < p->numObstacles; ++k)
    obs.push_back(make_float4(p->obstacles[k][0], p->obstacles[k][1], p->obstacles[k][2], p->obstacles[k][3]));
  if (!obs.empty())
    BRT_CUDA_TRY(cudaMemcpyAsync(e->obstacles + d.obsBase, obs.data(), sizeof(float4) * obs.size(), cudaMemcpyHostToDevice, e->stream));
  std::vector<uint2> field;
  if (e->obsMask) {
    field.assign(e->C, make_uint2(0u, 0u));
    buildObstacleField(*p, d, field);
    BRT_CUDA_TRY(cudaMemcpyAsync(e->obsMask + d.cellBase, field.data() + d.cellBase, sizeof(uint2) * d.C,
                                 cudaMemcpyHostToDevice, e->stream));
  }
  BRT_CUDA_TRY(invalidateResort(e));
  BRT_CUDA_TRY(cudaStreamSynchronize(e->stream));
  for (auto& kv : e->graphs) cudaGraphExecDestroy(kv.second);
  e->graphs.clear();
  e->paramsVersion++;
  return BRT_OK;
}

int brt_engine_set_option(brt_engine* e, const char* key, int64_t value) {
  if (!e || !key) return brt::argError(__func__);
  DeviceGuard guard(e->device);
  const std::string k(key);
  if (k == "two_pass") {
    e->forceTwoPass = value != 0;
  } else if (k == "phase2_variant") {
    if (value < 0 || value > 2) { setLastError("phase2_variant must be in [0, 2]"); return BRT_ERR_ARG; }
    e->phase2Variant = (int)value;
  } else if (k == "scan_variant") {
    if (value < 0 || value > 7) { setLastError("scan_variant must be in [0, 7]"); return BRT_ERR_ARG; }
    e->scanVariant = (int)value;
  } else if (k == "incremental_sort") {
    e->resortOn = value != 0;
    BRT_CUDA_TRY(invalidateResort(e));
  } else if (k == "block_size") {
    if (value < 32 || value > (int64_t)kFlockMaxThreads || value % 32) {
      setLastError("block_size must be a multiple of 32 in [32, 256]");
      return BRT_ERR_ARG;
    }
    e->fusedBlock = (uint32_t)value;
  } else if (k == "random_step") {
    if (value < 0 || value > 0xFFFFFFFFll) { setLastError("random_step must be a uint32"); return BRT_ERR_ARG; }
    const uint32_t v = (uint32_t)value;
    BRT_CUDA_TRY(cudaMemcpyAsync(e->stepCounter, &v, 4, cudaMemcpyHostToDevice, e->stream));
    BRT_CUDA_TRY(cudaStreamSynchronize(e->stream));
    return BRT_OK;  // a value, not a launch configuration: graphs stay valid
  } else if (k == "wide_registers") {
    e->regBudget = value != 0 ? 128 : 64;
  } else if (k == "registers") {
    if (value != 128 && value != 64 && value != 48 && value != 40) {
      setLastError("registers must be 128, 64, 48 or 40");
      return BRT_ERR_ARG;
    }
    e->regBudget = (int)value;
  } else if (k == "adjoint_graphs") {
    e->adjointGraphs = value != 0;
  } else if (k == "adjoint_export") {
    e->adjointExport = value != 0;
  } else if (k == "lookback_spin_limit") {
    if (value < 0 || value > 0x7FFFFFFFll) { setLastError("lookback_spin_limit must be in [0, 2^31)"); return BRT_ERR_ARG; }
    e->wait.spinLimit = (uint32_t)value;
    e->plan.wait = e->wait;
  } else if (k == "lookback_stall_tile") {
    if (value < -1 || value > 0x7FFFFFFFll) { setLastError("lookback_stall_tile must be -1 or a tile index"); return BRT_ERR_ARG; }
    e->wait.stallTile = value < 0 ? kNoStallTile : (uint32_t)value;
    e->plan.wait = e->wait;
  } else if (k == "sort_digit_bits") {
    if (value < 4 || value > 9) { setLastError("sort_digit_bits must be in [4, 9]"); return BRT_ERR_ARG; }
    BRT_CUDA_TRY(cudaStreamSynchronize(e->stream));
    SortPlan plan = makeSortPlan(e->N, e->plan.bits, (uint32_t)value);
    plan.wait = e->wait;
    const size_t bytes = sortScratchBytes(plan, false);
    void* mem = nullptr;
    BRT_CUDA_TRY(cudaMalloc(&mem, bytes));
    BRT_CUDA_TRY(cudaMemset(mem, 0, bytes));
    if (e->sortMem) cudaFree(e->sortMem);
    e->sortMem = mem;
    e->plan = plan;
    e->ss = carveSortScratch(plan, mem, false);
    e->reordered = false;
    e->listsValid = false;
    BRT_CUDA_TRY(invalidateResort(e));
  } else {
    setLastError("unknown option " + k);
    return BRT_ERR_ARG;
  }
  for (auto& kv : e->graphs) cudaGraphExecDestroy(kv.second);
  e->graphs.clear();
  e->paramsVersion++;
  return BRT_OK;
}

int brt_engine_stream(brt_engine* e, void** stream) {
  if (!e || !stream) return brt::argError(__func__);
  *stream = (void*)e->stream;
  return BRT_OK;
}

int brt_sync(brt_engine* e) {
  if (!e) return brt::argError(__func__);
  DeviceGuard guard(e->device);
  return syncAndCheck(e);
}

int brt_engine_record_lists(brt_engine* e, int enable) {
  if (!e) return brt::argError(__func__);
  e->recordLists = enable != 0;
  return BRT_OK;
}

int brt_engine_check_device_error(brt_engine* e, uint32_t* word) {
  if (!e || !word) return brt::argError(__func__);
  DeviceGuard guard(e->device);
  BRT_CUDA_TRY(cudaMemcpyAsync(word, e->errWord, 4, cudaMemcpyDeviceToHost, e->stream));
  BRT_CUDA_TRY(cudaStreamSynchronize(e->stream));
  if (*word) e->stateLost = true;
  BRT_CUDA_TRY(cudaMemsetAsync(e->errWord, 0, 4, e->stream));
  BRT_CUDA_TRY(cudaStreamSynchronize(e->stream));
  return BRT_OK;
}

// ---- feature I/O ------------------------------------------------------------

int brt_set_state(brt_engine* e, const float* pos4, const float* fwd4, const float* acc4, const float* features, int where) {
  brt::TraceRange trace(__func__);
  if (!e) return brt::argError(__func__);
  if (where != BRT_MEM_HOST && where != BRT_MEM_DEVICE) return brt::argError(__func__);
  DeviceGuard guard(e->device);
  cudaStream_t st = e->stream;
  const size_t n = e->N;
  if (e->stateLost && n) {
    // After a failed device check the slot order may hold an agent twice:
    // start again from the identity order (registered arrays included,
    // whose contents the caller sets again) and a clean re-sort state.
    BRT_CUDA_TRY(launchIota(e->idA, e->N, st));
    if (e->userIds.a) BRT_CUDA_TRY(launchIota(e->userIds.a, e->N, st));
    // a garbled order can leave mover lists of cells that end up empty
    BRT_CUDA_TRY(resetResort(e));
    e->stateLost = false;
  }
  auto stage4 = [&](const float* src) -> const float4* {
    if (where == BRT_MEM_DEVICE) return (const float4*)src;
    cudaMemcpyAsync(e->stage4, src, n * 16, cudaMemcpyHostToDevice, st);
    return e->stage4;
  };
  if (n == 0) return BRT_OK;
  // Inputs are in agent-id order; the canonical arrays are in slot order.
  if (pos4) { const float4* s = stage4(pos4); BRT_CUDA_TRY(launchGatherFromId(s, e->idA, e->posA, e->N, true, st)); }
  if (fwd4) { const float4* s = stage4(fwd4); BRT_CUDA_TRY(launchGatherFromId(s, e->idA, e->fwdA, e->N, false, st)); }
  if (acc4) { const float4* s = stage4(acc4); BRT_CUDA_TRY(launchGatherFromId(s, e->idA, e->accA, e->N, false, st)); }
  if (features && e->Fmax) {
    const float* s = features;
    if (where == BRT_MEM_HOST) {
      BRT_CUDA_TRY(cudaMemcpyAsync(e->stageF, features, n * e->Fmax * 4, cudaMemcpyHostToDevice, st));
      s = e->stageF;
    }
    BRT_CUDA_TRY(launchGatherFeatFromId(s, e->Fmax, e->idA, e->featA, e->Fs, e->N, st));
  }
  e->reordered = false;
  e->listsValid = false;
  BRT_CUDA_TRY(invalidateResort(e));
  if (where == BRT_MEM_HOST) BRT_CUDA_TRY(cudaStreamSynchronize(st));
  return BRT_OK;
}

int brt_get_state(brt_engine* e, float* pos4, float* fwd4, float* acc4, float* features, int where) {
  brt::TraceRange trace(__func__);
  if (!e) return brt::argError(__func__);
  if (where != BRT_MEM_HOST && where != BRT_MEM_DEVICE) return brt::argError(__func__);
  DeviceGuard guard(e->device);
  cudaStream_t st = e->stream;
  const size_t n = e->N;
  if (n == 0) return BRT_OK;
  float4* srcs[3] = {e->posA, e->fwdA, e->accA};
  float* dsts[3] = {pos4, fwd4, acc4};
  for (int k = 0; k < 3; ++k) {
    if (!dsts[k]) continue;
    if (where == BRT_MEM_DEVICE) {
      BRT_CUDA_TRY(launchScatterToId(srcs[k], e->idA, (float4*)dsts[k], e->N, st));
    } else {
      BRT_CUDA_TRY(launchScatterToId(srcs[k], e->idA, e->stage4, e->N, st));
      BRT_CUDA_TRY(cudaMemcpyAsync(dsts[k], e->stage4, n * 16, cudaMemcpyDeviceToHost, st));
    }
  }
  if (features && e->Fmax) {
    if (where == BRT_MEM_DEVICE) {
      BRT_CUDA_TRY(launchScatterFeatToId(e->featA, e->Fs, e->idA, features, e->Fmax, e->N, st));
    } else {
      BRT_CUDA_TRY(launchScatterFeatToId(e->featA, e->Fs, e->idA, e->stageF, e->Fmax, e->N, st));
      BRT_CUDA_TRY(cudaMemcpyAsync(features, e->stageF, n * e->Fmax * 4, cudaMemcpyDeviceToHost, st));
    }
  }
  if (where == BRT_MEM_HOST) return syncAndCheck(e);
  return BRT_OK;
}

int brt_set_similarity_stats(brt_engine* e, const float* stats4, int where) {
  if (!e || !stats4) return brt::argError(__func__);
  DeviceGuard guard(e->device);
  BRT_CUDA_TRY(cudaMemcpyAsync(e->statsById, stats4, (size_t)e->N * 16,
                               where == BRT_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, e->stream));
  if (where == BRT_MEM_HOST) BRT_CUDA_TRY(cudaStreamSynchronize(e->stream));
  return BRT_OK;
}

int brt_get_similarity_stats(brt_engine* e, float* stats4, int where) {
  if (!e || !stats4) return brt::argError(__func__);
  DeviceGuard guard(e->device);
  BRT_CUDA_TRY(cudaMemcpyAsync(stats4, e->statsById, (size_t)e->N * 16,
                               where == BRT_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, e->stream));
  if (where == BRT_MEM_HOST) return syncAndCheck(e);
  return BRT_OK;
}

// ---- fused step --------------------------------------------------------------

int brt_step(brt_engine* e, float elapsedTime, uint32_t nsteps) {
  brt::TraceRange trace(__func__);
  if (!e) return brt::argError(__func__);
  if (nsteps == 0 || e->N == 0) return BRT_OK;
  DeviceGuard guard(e->device);
  const bool record = e->recordLists;
  if (nsteps == 1) {
    int rc = enqueueStep(e, elapsedTime, record);
    if (rc) return rc;
  } else {
    cudaGraphExec_t ge = nullptr;
    int rc = getGraph(e, elapsedTime, nsteps, record, &ge);
    if (rc) return rc;
    BRT_CUDA_TRY(cudaGraphLaunch(ge, e->stream));
  }
  e->reordered = true;
  e->listsValid = record;
  return BRT_OK;
}

int brt_step_prepare(brt_engine* e, float elapsedTime, uint32_t nsteps) {
  brt::TraceRange trace(__func__);
  if (!e) return brt::argError(__func__);
  if (nsteps < 2 || e->N == 0) return BRT_OK;
  DeviceGuard guard(e->device);
  cudaGraphExec_t ge = nullptr;
  return getGraph(e, elapsedTime, nsteps, e->recordLists, &ge);
}

int brt_engine_stage_timing(brt_engine* e, int enable) {
  if (!e) return brt::argError(__func__);
  DeviceGuard guard(e->device);
  if (enable && !e->ev[0][0]) {
    for (int r = 0; r < brt_engine::kRing; ++r)
      for (int k = 0; k < 5; ++k) BRT_CUDA_TRY(cudaEventCreate(&e->ev[r][k]));
  }
  if (!enable) {
    for (int r = 0; r < brt_engine::kRing; ++r) {
      int rc = drainSlot(e, r);
      if (rc) return rc;
    }
  }
  e->timing = enable != 0;
  return BRT_OK;
}

int brt_engine_stage_times(brt_engine* e, double* ms4, uint64_t* steps, uint32_t* launches_per_step) {
  if (!e) return brt::argError(__func__);
  DeviceGuard guard(e->device);
  for (int r = 0; r < brt_engine::kRing; ++r) {
    int rc = drainSlot(e, (e->ringPos + r) % brt_engine::kRing);
    if (rc) return rc;
  }
  if (ms4) for (int k = 0; k < 4; ++k) ms4[k] = e->stageMs[k];
  if (steps) *steps = e->timedSteps;
  // hash, radix passes, reorder, flock; with the incremental re-sort also its
  // mark, cell-scan and place kernels (the hash and the passes still launch
  // and return at once on the steps they are not needed)
  if (launches_per_step) *launches_per_step = 3 + e->plan.passes + (e->resortOn ? 3 : 0);
  e->stageMs[0] = e->stageMs[1] = e->stageMs[2] = e->stageMs[3] = 0;
  e->timedSteps = 0;
  return BRT_OK;
}

int brt_engine_autotune(brt_engine* e, float elapsedTime, uint32_t steps, char* report, size_t report_len) {
  brt::TraceRange trace(__func__);
  if (!e || steps == 0) return brt::argError(__func__);
  if (e->N == 0) return BRT_OK;
  DeviceGuard guard(e->device);
  cudaStream_t st = e->stream;
  const size_t n = e->N;
  BRT_CUDA_TRY(cudaStreamSynchronize(st));
  // Snapshot of the canonical state: every trial starts from it, and the
  // engine is left in it.
  float4 *sp = nullptr, *sf = nullptr, *sa = nullptr, *ss = nullptr;
  uint32_t* si = nullptr;
  float* sx = nullptr;
  int rc = BRT_OK;
  auto chk = [&](int r) { if (r && !rc) rc = r; };
  chk(devAlloc(&sp, n)); chk(devAlloc(&sf, n)); chk(devAlloc(&sa, n)); chk(devAlloc(&ss, n)); chk(devAlloc(&si, n));
  chk(devAlloc(&sx, n * e->Fs));
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  if (!rc && (cudaEventCreate(&t0) != cudaSuccess || cudaEventCreate(&t1) != cudaSuccess)) {
    setLastError("event creation failed");
    rc = BRT_ERR_CUDA;
  }
  auto copyAll = [&](bool save) -> cudaError_t {
    cudaError_t c = cudaSuccess;
    auto cp = [&](void* dst, const void* src, size_t bytes) {
      if (c == cudaSuccess && bytes) c = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st);
    };
    if (save) {
      cp(sp, e->posA, n * 16); cp(sf, e->fwdA, n * 16); cp(sa, e->accA, n * 16); cp(ss, e->statsById, n * 16);
      cp(si, e->idA, n * 4); cp(sx, e->featA, n * e->Fs * 4);
    } else {
      cp(e->posA, sp, n * 16); cp(e->fwdA, sf, n * 16); cp(e->accA, sa, n * 16); cp(e->statsById, ss, n * 16);
      cp(e->idA, si, n * 4); cp(e->featA, sx, n * e->Fs * 4);
      if (c == cudaSuccess) c = invalidateResort(e);
    }
    return c;
  };
  if (!rc && copyAll(true) != cudaSuccess) { setLastError("autotune snapshot failed"); rc = BRT_ERR_CUDA; }
  // The trials' steps are undone, so registered arrays stay where they are;
  // graphs captured while frozen are keyed apart from the others.
  const bool wasFrozen = e->userFrozen;
  e->userFrozen = true;
  e->paramsVersion++;
  // One trial: the steps-step graph launched twice from the snapshot, the
  // faster launch counted.
  auto measure = [&](double* msPerStep) -> int {
    cudaGraphExec_t ge = nullptr;
    int r = getGraph(e, elapsedTime, steps, false, &ge);
    if (r) return r;
    double best = 1e30;
    for (int rep = 0; rep < 2; ++rep) {
      BRT_CUDA_TRY(copyAll(false));
      BRT_CUDA_TRY(cudaEventRecord(t0, st));
      BRT_CUDA_TRY(cudaGraphLaunch(ge, st));
      BRT_CUDA_TRY(cudaEventRecord(t1, st));
      BRT_CUDA_TRY(cudaEventSynchronize(t1));
      float ms = 0.0f;
      BRT_CUDA_TRY(cudaEventElapsedTime(&ms, t0, t1));
      best = std::min(best, (double)ms / steps);
    }
    if ((r = checkDeviceError(e, true))) return r;
    *msPerStep = best;
    return BRT_OK;
  };
  // The flock kernel's options only matter when that kernel runs.
  bool twoPass = e->anyKnn || e->forceTwoPass || e->school;
  for (const FlockDev& d : e->flocksHost) twoPass = twoPass || (d.F > 0 && (d.clus != 0.0f || d.aclus != 0.0f));
  std::string log;
  char buf[256];
  auto trial = [&](const char* what, int64_t v, double* ms) -> int {
    int r = measure(ms);
    std::snprintf(buf, sizeof(buf), "%s{\"%s\": %lld, \"ms_per_step\": %.6f}", log.empty() ? "" : ", ", what, (long long)v, *ms);
    log += buf;
    return r;
  };
  // Coordinate descent: radix digit width, then block size x scan loop
  // shape, then the list-walk variant (the last two only when the
  // single-pass kernel runs).
  uint32_t bestBits = e->plan.digitBits;
  double bestMs = 1e30, ms = 0.0;
  // digit widths are timed with the full sort every step (the incremental
  // re-sort would hide them)
  const bool resortWas = e->resortOn;
  e->resortOn = false;
  for (uint32_t b = 4; b <= 8 && !rc; ++b) {
    chk(brt_engine_set_option(e, "sort_digit_bits", b));
    if (!rc) chk(trial("sort_digit_bits", b, &ms));
    if (!rc && ms < bestMs) { bestMs = ms; bestBits = b; }
  }
  e->resortOn = resortWas;
  if (!rc) chk(brt_engine_set_option(e, "sort_digit_bits", bestBits));
  uint32_t bestBlock = e->fusedBlock;
  int bestScan = e->scanVariant, bestP2 = e->phase2Variant;
  int bestRegs = e->regBudget;
  if (!twoPass) {
    bestMs = 1e30;
    // block size x scan loop x list walk, jointly: the best block depends on
    // the walk.  Walk 1 (two neighbours at a time) only exists for the
    // per-agent scans, walk 2 (geometry, then feature sums) for the
    // cooperative scan of flocks with features.
    const uint32_t blocks[3] = {64, 128, 256};
    // per agent with / without cell culling, warp-cooperative, cooperative
    // with windows, cooperative with bounding-box culling
    const int scans[5] = {0, 2, 4, 5, 7};
    const char* names[5][2] = {{"block_size/scan0/walk0", "block_size/scan0/walk1"},
                               {"block_size/scan2/walk0", "block_size/scan2/walk1"},
                               {"block_size/scan4/walk0", "block_size/scan4/walk2"},
                               {"block_size/scan5/walk0", "block_size/scan5/walk2"},
                               {"block_size/scan7/walk0", "block_size/scan7/walk2"}};
    bool anyFeatures = false;
    for (const FlockDev& d : e->flocksHost) anyFeatures = anyFeatures || (d.F > 0 && d.relax != 0.0f);
    for (uint32_t bs : blocks)
      for (int s = 0; s < 5 && !rc; ++s)
        for (int w = 0; w < 2 && !rc; ++w) {
          const int p2 = w == 0 ? 0 : (scans[s] >= 4 ? 2 : 1);
          if (p2 == 2 && !anyFeatures) continue;
          chk(brt_engine_set_option(e, "block_size", bs));
          chk(brt_engine_set_option(e, "scan_variant", scans[s]));
          chk(brt_engine_set_option(e, "phase2_variant", p2));
          if (!rc) chk(trial(names[s][w], bs, &ms));
          if (!rc && ms < bestMs) { bestMs = ms; bestBlock = bs; bestScan = scans[s]; bestP2 = p2; }
        }
    // the staged tile kernel (its block is fixed)
    for (int w = 0; w < 2 && !rc; ++w) {
      const int p2 = w == 0 ? 0 : 2;
      if (p2 == 2 && !anyFeatures) continue;
      chk(brt_engine_set_option(e, "scan_variant", 6));
      chk(brt_engine_set_option(e, "phase2_variant", p2));
      if (!rc) chk(trial(w == 0 ? "scan6/walk0" : "scan6/walk2", kTileThreads, &ms));
      if (!rc && ms < bestMs) { bestMs = ms; bestScan = 6; bestP2 = p2; }
    }
    if (!rc) {
      chk(brt_engine_set_option(e, "block_size", bestBlock));
      chk(brt_engine_set_option(e, "scan_variant", bestScan));
      chk(brt_engine_set_option(e, "phase2_variant", bestP2));
    }
    // 48 and 40 only change the cooperative scan's build; the tile kernel has one
    const int budgets[4] = {64, 128, 48, 40};
    const int nBudgets = bestScan == 6 ? 0 : (bestScan >= 4 ? 4 : 2);
    bestMs = 1e30;
    for (int r = 0; r < nBudgets && !rc; ++r) {
      chk(brt_engine_set_option(e, "registers", budgets[r]));
      if (!rc) chk(trial("registers", (uint32_t)budgets[r], &ms));
      if (!rc && ms < bestMs) { bestMs = ms; bestRegs = budgets[r]; }
    }
    if (!rc) chk(brt_engine_set_option(e, "registers", bestRegs));
  }
  // the incremental re-sort against the full sort every step
  {
    const int start = e->resortOn ? 1 : 0;
    int bestResort = start;
    bestMs = 1e30;
    for (int k = 0; k < 2 && !rc; ++k) {
      const int v = k == 0 ? start : 1 - start;
      chk(brt_engine_set_option(e, "incremental_sort", v));
      if (!rc) chk(trial("incremental_sort", (uint32_t)v, &ms));
      if (!rc && ms < bestMs) { bestMs = ms; bestResort = v; }
    }
    if (!rc) chk(brt_engine_set_option(e, "incremental_sort", bestResort));
  }
  if (!rc && copyAll(false) != cudaSuccess) { setLastError("autotune restore failed"); rc = BRT_ERR_CUDA; }
  if (!rc) cudaStreamSynchronize(st);
  e->userFrozen = wasFrozen;
  e->paramsVersion++;
  e->reordered = false;
  e->listsValid = false;
  if (t0) cudaEventDestroy(t0);
  if (t1) cudaEventDestroy(t1);
  for (void* p : {(void*)sp, (void*)sf, (void*)sa, (void*)ss, (void*)si, (void*)sx})
    if (p) cudaFree(p);
  if (rc) return rc;
  if (report && report_len) {
    std::snprintf(buf, sizeof(buf),
                  "{\"sort_digit_bits\": %u, \"block_size\": %u, \"scan_variant\": %d, \"phase2_variant\": %d, "
                  "\"wide_registers\": %d, \"registers\": %d, \"incremental_sort\": %d, \"ms_per_step\": %.6f, "
                  "\"trials\": [",
                  bestBits, bestBlock, bestScan, bestP2, bestRegs > 64 ? 1 : 0, bestRegs, e->resortOn ? 1 : 0, bestMs);
    std::string out = std::string(buf) + log + "]}";
    std::snprintf(report, report_len, "%s", out.c_str());
  }
  return BRT_OK;
}

// ---- stage-wise functionalities ------------------------------------------------

int brt_reorder_sim_data(brt_engine* e) {
  brt::TraceRange trace(__func__);
  if (!e) return brt::argError(__func__);
  DeviceGuard guard(e->device);
  if (e->N == 0) return BRT_OK;
  int rc = enqueueReorder(e);
  if (rc) return rc;
  e->reordered = true;
  e->listsValid = false;
  return BRT_OK;
}

int brt_compute_neighborhoods(brt_engine* e) {
  brt::TraceRange trace(__func__);
  if (!e) return brt::argError(__func__);
  if (!e->reordered) { setLastError("computeNeighborhoods before reorderSimData"); return BRT_ERR_STATE; }
  DeviceGuard guard(e->device);
  BRT_CUDA_TRY(launchLists(stageArgs(e), e->anyKnn, e->stream));
  e->listsValid = true;
  return BRT_OK;
}

int brt_reset_steer_force(brt_engine* e) {
  brt::TraceRange trace(__func__);
  if (!e) return brt::argError(__func__);
  DeviceGuard guard(e->device);
  if (e->N) BRT_CUDA_TRY(cudaMemsetAsync(e->steer, 0, (size_t)e->N * 16, e->stream));
  return BRT_OK;
}

static int steerStage(brt_engine* e, int which) {
  if (!e) return brt::argError(__func__);
  if (!e->reordered || !e->listsValid) { setLastError("steering stage before computeNeighborhoods"); return BRT_ERR_STATE; }
  DeviceGuard guard(e->device);
  BRT_CUDA_TRY(launchSteerStage(stageArgs(e), which, e->stream));
  return BRT_OK;
}

int brt_compute_separations(brt_engine* e) {
  brt::TraceRange trace(__func__);
  return steerStage(e, 0);
}
int brt_compute_alignments(brt_engine* e) {
  brt::TraceRange trace(__func__);
  return steerStage(e, 1);
}
int brt_compute_cohesions(brt_engine* e) {
  brt::TraceRange trace(__func__);
  return steerStage(e, 2);
}
int brt_steer_for_clustering(brt_engine* e) {
  brt::TraceRange trace(__func__);
  return steerStage(e, 3);
}
// In the periodic world every position is inside the world box, so the
// reference's seek-to-centre force is zero (OpenSteerWrapper_kernel.cu:236-246);
// this stage applies the static obstacle field of the EnvGrid3D grid instead.
int brt_compute_seekings_world_center(brt_engine* e) {
  brt::TraceRange trace(__func__);
  return steerStage(e, 4);
}
int brt_steer_and_slow_to_avoid_neighbors(brt_engine* e) {
  brt::TraceRange trace(__func__);
  return steerStage(e, 5);
}
int brt_steer_for_move_away_base_target(brt_engine* e, const float* base3, const float* params3) {
  brt::TraceRange trace(__func__);
  if (!e || !base3) return brt::argError(__func__);
  if (!e->reordered || !e->listsValid) { setLastError("steering stage before computeNeighborhoods"); return BRT_ERR_STATE; }
  DeviceGuard guard(e->device);
  StageArgs A = stageArgs(e);
  // OpenSteerWrapperPlugIn.h:144-150: (500, 500, 1000) when the weight is 0
  const float defaults[3] = {500.0f, 500.0f, 1000.0f};
  const float* p = (params3 && params3[0] != 0.0f) ? params3 : defaults;
  for (int k = 0; k < 3; ++k) {
    A.avoidBase[k] = base3[k];
    A.avoidBaseParams[k] = p[k];
  }
  BRT_CUDA_TRY(launchSteerStage(A, 6, e->stream));
  return BRT_OK;
}

// ---- on-disk state snapshot ----------------------------------------------------

namespace {
constexpr char kSnapMagic[8] = {'B', 'R', 'T', 'S', 'N', 'A', 'P', '1'};
struct SnapHeader {
  char magic[8];
  uint32_t version, n, features, nflocks, step, reserved[3];
};
}  // namespace

int brt_save_snapshot(brt_engine* e, const char* path) {
  brt::TraceRange trace(__func__);
  if (!e || !path) return brt::argError(__func__);
  DeviceGuard guard(e->device);
  const size_t n = e->N, F = e->Fmax;
  std::vector<float> pos(4 * n), fwd(4 * n), acc(4 * n), stats(4 * n), feat(n * F);
  int rc = brt_get_state(e, pos.data(), fwd.data(), acc.data(), F ? feat.data() : nullptr, BRT_MEM_HOST);
  if (rc) return rc;
  if ((rc = brt_get_similarity_stats(e, stats.data(), BRT_MEM_HOST))) return rc;
  SnapHeader h;
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.magic, kSnapMagic, 8);
  h.version = 1; h.n = e->N; h.features = e->Fmax; h.nflocks = e->nflocks;
  BRT_CUDA_TRY(cudaMemcpyAsync(&h.step, e->stepCounter, 4, cudaMemcpyDeviceToHost, e->stream));
  BRT_CUDA_TRY(cudaStreamSynchronize(e->stream));
  FILE* f = std::fopen(path, "wb");
  if (!f) { setLastError(std::string("cannot open ") + path + " for writing"); return BRT_ERR_ARG; }
  bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1;
  for (const std::vector<float>* v : {&pos, &fwd, &acc, &stats, &feat})
    ok = ok && (v->empty() || std::fwrite(v->data(), 4, v->size(), f) == v->size());
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) { setLastError(std::string("writing ") + path + " failed"); return BRT_ERR_ARG; }
  return BRT_OK;
}

int brt_load_snapshot(brt_engine* e, const char* path) {
  brt::TraceRange trace(__func__);
  if (!e || !path) return brt::argError(__func__);
  DeviceGuard guard(e->device);
  FILE* f = std::fopen(path, "rb");
  if (!f) { setLastError(std::string("cannot open ") + path); return BRT_ERR_ARG; }
  SnapHeader h;
  bool ok = std::fread(&h, sizeof(h), 1, f) == 1 && std::memcmp(h.magic, kSnapMagic, 8) == 0 && h.version == 1;
  if (ok && (h.n != e->N || h.features != e->Fmax || h.nflocks != e->nflocks)) {
    std::fclose(f);
    setLastError("snapshot does not match the engine (agents, features or flocks differ)");
    return BRT_ERR_CONFIG;
  }
  const size_t n = e->N, F = e->Fmax;
  std::vector<float> pos(4 * n), fwd(4 * n), acc(4 * n), stats(4 * n), feat(n * F);
  for (std::vector<float>* v : {&pos, &fwd, &acc, &stats, &feat})
    ok = ok && (v->empty() || std::fread(v->data(), 4, v->size(), f) == v->size());
  std::fclose(f);
  if (!ok) { setLastError(std::string(path) + " is not a complete snapshot"); return BRT_ERR_ARG; }
  int rc = brt_set_state(e, pos.data(), fwd.data(), acc.data(), F ? feat.data() : nullptr, BRT_MEM_HOST);
  if (rc) return rc;
  if ((rc = brt_set_similarity_stats(e, stats.data(), BRT_MEM_HOST))) return rc;
  BRT_CUDA_TRY(cudaMemcpyAsync(e->stepCounter, &h.step, 4, cudaMemcpyHostToDevice, e->stream));
  BRT_CUDA_TRY(cudaStreamSynchronize(e->stream));
  return BRT_OK;
}

// ---- BehaviorClustering analytics --------------------------------------------

static ClusterArgs clusterArgs(brt_engine* e, float radius) {
  ClusterArgs A;
  std::memset(&A, 0, sizeof(A));
  A.posS = e->posS; A.idS = e->idS; A.lists = e->lists; A.listStride = e->listStride;
  A.flocks = e->flocks; A.agentBase = e->agentBase; A.nflocks = e->nflocks; A.n = e->N;
  A.radius = radius;
  A.in = e->membership[e->membershipCur];
  A.out = e->membership[e->membershipCur ^ 1];
  return A;
}

static int clusterReady(brt_engine* e) {
  if (!e->listsValid) {
    setLastError("cluster analytics need the neighbour lists (computeNeighborhoods or record_lists)");
    return BRT_ERR_STATE;
  }
  for (int k = 0; k < 2 && !e->membership[k]; ++k) {
    int rc = devAlloc(&e->membership[k], e->N);
    if (rc) return rc;
    BRT_CUDA_TRY(cudaMemsetAsync(e->membership[k], 0, (size_t)e->N * 16, e->stream));
  }
  return BRT_OK;
}

int brt_compute_cluster_membership(brt_engine* e, uint32_t iterations) {
  brt::TraceRange trace(__func__);
  if (!e) return brt::argError(__func__);
  DeviceGuard guard(e->device);
  int rc = clusterReady(e);
  if (rc || e->N == 0) return rc;
  for (uint32_t it = 0; it <= iterations; ++it) {
    BRT_CUDA_TRY(launchCluster(clusterArgs(e, 0.0f), it == 0 ? 0 : 1, e->stream));
    e->membershipCur ^= 1;
  }
  return BRT_OK;
}

int brt_analyze_cluster_hit_rate(brt_engine* e, float same_cluster_max_radius) {
  brt::TraceRange trace(__func__);
  if (!e) return brt::argError(__func__);
  DeviceGuard guard(e->device);
  int rc = clusterReady(e);
  if (rc || e->N == 0) return rc;
  BRT_CUDA_TRY(launchCluster(clusterArgs(e, same_cluster_max_radius), 2, e->stream));
  e->membershipCur ^= 1;
  return BRT_OK;
}

int brt_get_cluster_membership(brt_engine* e, float* membership4, int where) {
  if (!e || !membership4) return brt::argError(__func__);
  if (!e->membership[0]) { setLastError("no cluster membership computed yet"); return BRT_ERR_STATE; }
  DeviceGuard guard(e->device);
  BRT_CUDA_TRY(cudaMemcpyAsync(membership4, e->membership[e->membershipCur], (size_t)e->N * 16,
                               where == BRT_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, e->stream));
  if (where == BRT_MEM_HOST) return syncAndCheck(e);
  return BRT_OK;
}

static int schoolStage(brt_engine* e, int which) {
  if (!e) return brt::argError(__func__);
  if (!e->school) { setLastError("Schooling functionality on a flocking engine (schooling.mode 0)"); return BRT_ERR_STATE; }
  if (!e->reordered || !e->listsValid) { setLastError("Schooling functionality before computeNeighborhoods"); return BRT_ERR_STATE; }
  DeviceGuard guard(e->device);
  BRT_CUDA_TRY(launchSchoolStage(stageArgs(e), which, e->stream));
  return BRT_OK;
}

int brt_school_repulsion(brt_engine* e) {
  brt::TraceRange trace(__func__);
  return schoolStage(e, 0);
}
int brt_school_attraction_orientation(brt_engine* e) {
  brt::TraceRange trace(__func__);
  return schoolStage(e, 1);
}
int brt_school_movement(brt_engine* e) {
  brt::TraceRange trace(__func__);
  return schoolStage(e, 2);
}
int brt_school_animate(brt_engine* e) {
  brt::TraceRange trace(__func__);
  return schoolStage(e, 3);
}

int brt_apply_steering_forces(brt_engine* e, float elapsedTime) {
  brt::TraceRange trace(__func__);
  if (!e) return brt::argError(__func__);
  if (!e->reordered || !e->listsValid) { setLastError("applySteeringForces before computeNeighborhoods"); return BRT_ERR_STATE; }
  DeviceGuard guard(e->device);
  BRT_CUDA_TRY(launchIntegrateStage(stageArgs(e), elapsedTime, e->stream));
  return BRT_OK;
}

// ---- getters -------------------------------------------------------------------

static cudaMemcpyKind kindOut(int where) { return where == BRT_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice; }

int brt_get_hash(brt_engine* e, uint32_t* keys, uint32_t* ids, int where) {
  if (!e) return brt::argError(__func__);
  if (!e->reordered) { setLastError("getHash before reorderSimData"); return BRT_ERR_STATE; }
  DeviceGuard guard(e->device);
  const size_t n = e->N;
  if (n == 0) return BRT_OK;
  if (where == BRT_MEM_DEVICE) {
    BRT_CUDA_TRY(launchHashPairsOut(e->pairs[e->finalPairs], e->idS, keys, ids, e->N, e->stream));
    return BRT_OK;
  }
  uint32_t* tk = (uint32_t*)e->stage4;
  uint32_t* ti = tk + n;
  BRT_CUDA_TRY(launchHashPairsOut(e->pairs[e->finalPairs], e->idS, tk, ti, e->N, e->stream));
  if (keys) BRT_CUDA_TRY(cudaMemcpyAsync(keys, tk, n * 4, cudaMemcpyDeviceToHost, e->stream));
  if (ids) BRT_CUDA_TRY(cudaMemcpyAsync(ids, ti, n * 4, cudaMemcpyDeviceToHost, e->stream));
  return syncAndCheck(e);
}

int brt_get_cell_ranges(brt_engine* e, uint32_t* cell_start, uint32_t* cell_end, int where) {
  if (!e) return brt::argError(__func__);
  if (!e->reordered) { setLastError("getCellStart before reorderSimData"); return BRT_ERR_STATE; }
  DeviceGuard guard(e->device);
  if (cell_start) BRT_CUDA_TRY(cudaMemcpyAsync(cell_start, e->cellStart, (size_t)e->C * 4, kindOut(where), e->stream));
  if (cell_end) BRT_CUDA_TRY(cudaMemcpyAsync(cell_end, e->cellEnd, (size_t)e->C * 4, kindOut(where), e->stream));
  if (where == BRT_MEM_HOST) return syncAndCheck(e);
  return BRT_OK;
}

int brt_get_neighbor_lists(brt_engine* e, uint32_t* lists, int where) {
  if (!e || !lists) return brt::argError(__func__);
  if (!e->listsValid) { setLastError("neighbour lists not computed (computeNeighborhoods or record_lists)"); return BRT_ERR_STATE; }
  DeviceGuard guard(e->device);
  BRT_CUDA_TRY(cudaMemcpyAsync(lists, e->lists, (size_t)e->N * e->listStride * 4, kindOut(where), e->stream));
  if (where == BRT_MEM_HOST) return syncAndCheck(e);
  return BRT_OK;
}

int brt_get_steer_force(brt_engine* e, float* steer4, int where) {
  if (!e || !steer4) return brt::argError(__func__);
  DeviceGuard guard(e->device);
  BRT_CUDA_TRY(cudaMemcpyAsync(steer4, e->steer, (size_t)e->N * 16, kindOut(where), e->stream));
  if (where == BRT_MEM_HOST) return syncAndCheck(e);
  return BRT_OK;
}

// ---- plugin extension: registered arrays, the array view, user launches ----------

int brt_engine_add_array(brt_engine* e, uint32_t bytes_per_agent, uint32_t* array_id) {
  if (!e || !array_id) return brt::argError(__func__);
  if (bytes_per_agent == 0 || bytes_per_agent % 4 || bytes_per_agent > 1024) {
    setLastError("bytes_per_agent must be a multiple of 4 in [4, 1024]");
    return BRT_ERR_ARG;
  }
  if (e->user.size() >= BRT_MAX_USER_ARRAYS) { setLastError("too many registered arrays"); return BRT_ERR_CAPACITY; }
  DeviceGuard guard(e->device);
  const size_t n = std::max<size_t>(e->N, 1);
  const uint32_t words = bytes_per_agent / 4;
  BRT_CUDA_TRY(cudaStreamSynchronize(e->stream));
  if (!e->userIds.a) {
    // the id map starts as the engine's current slot order
    BRT_CUDA_TRY(cudaMalloc(&e->userIds.a, n * 4));
    BRT_CUDA_TRY(cudaMalloc(&e->userIds.s, n * 4));
    e->userIds.words = 1;
    if (e->N) BRT_CUDA_TRY(cudaMemcpyAsync(e->userIds.a, e->idA, (size_t)e->N * 4, cudaMemcpyDeviceToDevice, e->stream));
  }
  brt_engine::UserArray u;
  u.words = words;
  BRT_CUDA_TRY(cudaMalloc(&u.a, n * words * 4));
  if (cudaMalloc(&u.s, n * words * 4) != cudaSuccess) {
    cudaFree(u.a);
    setLastError("out of device memory");
    return BRT_ERR_CUDA;
  }
  BRT_CUDA_TRY(cudaMemsetAsync(u.a, 0, n * words * 4, e->stream));
  if (words > e->userStageWords) {
    if (e->userStage) cudaFree(e->userStage);
    e->userStage = nullptr;
    e->userStageWords = 0;
    BRT_CUDA_TRY(cudaMalloc(&e->userStage, n * words * 4));
    e->userStageWords = words;
  }
  e->user.push_back(u);
  *array_id = (uint32_t)e->user.size() - 1;
  e->paramsVersion++;  // captured step graphs must now include the permutation
  BRT_CUDA_TRY(cudaStreamSynchronize(e->stream));
  return BRT_OK;
}

int brt_engine_array_set(brt_engine* e, uint32_t array_id, const void* src, int where) {
  if (!e || !src || array_id >= e->user.size()) return brt::argError(__func__);
  if (where != BRT_MEM_HOST && where != BRT_MEM_DEVICE) return brt::argError(__func__);
  DeviceGuard guard(e->device);
  const brt_engine::UserArray& u = e->user[array_id];
  const size_t bytes = (size_t)e->N * u.words * 4;
  if (!bytes) return BRT_OK;
  const uint32_t* s = (const uint32_t*)src;
  if (where == BRT_MEM_HOST) {
    BRT_CUDA_TRY(cudaMemcpyAsync(e->userStage, src, bytes, cudaMemcpyHostToDevice, e->stream));
    s = e->userStage;
  }
  // slot i holds agent userIds[i]
  BRT_CUDA_TRY(launchGatherWords(s, e->userIds.a, 1, u.a, u.words, e->N, e->stream));
  if (where == BRT_MEM_HOST) return syncAndCheck(e);
  return BRT_OK;
}

int brt_engine_array_get(brt_engine* e, uint32_t array_id, void* dst, int where) {
  if (!e || !dst || array_id >= e->user.size()) return brt::argError(__func__);
  if (where != BRT_MEM_HOST && where != BRT_MEM_DEVICE) return brt::argError(__func__);
  DeviceGuard guard(e->device);
  const brt_engine::UserArray& u = e->user[array_id];
  const size_t bytes = (size_t)e->N * u.words * 4;
  if (!bytes) return BRT_OK;
  uint32_t* d = where == BRT_MEM_HOST ? e->userStage : (uint32_t*)dst;
  BRT_CUDA_TRY(launchScatterWords(u.a, e->userIds.a, d, u.words, e->N, e->stream));
  if (where == BRT_MEM_HOST) {
    BRT_CUDA_TRY(cudaMemcpyAsync(dst, e->userStage, bytes, cudaMemcpyDeviceToHost, e->stream));
    return syncAndCheck(e);
  }
  return BRT_OK;
}

int brt_engine_get_arrays(brt_engine* e, brt_arrays* out) {
  if (!e || !out) return brt::argError(__func__);
  std::memset(out, 0, sizeof(*out));
  out->num_agents = e->N;
  out->num_cells = e->C;
  out->features_stride = e->Fs;
  out->list_stride = e->listStride;
  out->pos4 = (float*)e->posA; out->forward4 = (float*)e->fwdA; out->smooth_accel4 = (float*)e->accA;
  out->features = e->featA;
  out->agent_id = e->idA;
  out->sorted_pos4 = (float*)e->posS; out->sorted_forward4 = (float*)e->fwdS;
  out->sorted_smooth_accel4 = (float*)e->accS; out->sorted_features = e->featS;
  out->sorted_agent_id = e->idS;
  out->steer4 = (float*)e->steer;
  out->neighbor_lists = e->lists;
  out->cell_start = e->cellStart; out->cell_end = e->cellEnd;
  out->num_user = (uint32_t)e->user.size();
  for (size_t k = 0; k < e->user.size(); ++k) {
    out->user[k] = e->user[k].a;
    out->user_bytes[k] = e->user[k].words * 4;
  }
  out->user_agent_id = e->userIds.a;
  return BRT_OK;
}

int brt_engine_launch(brt_engine* e, brt_launch_fn fn, void* user_data) {
  brt::TraceRange trace(__func__);
  if (!e || !fn) return brt::argError(__func__);
  DeviceGuard guard(e->device);
  brt_arrays view;
  int rc = brt_engine_get_arrays(e, &view);
  if (rc) return rc;
  fn(user_data, (void*)e->stream, &view);
  BRT_CUDA_TRY(cudaGetLastError());
  return BRT_OK;
}

}  // extern "C"

namespace {
// The kernels' dynamic shared-memory limits are per device and per function,
// shared by every engine of the process: they follow the largest
// maxNeighbors any engine on the device has asked for, so an engine created
// later with shorter lists never lowers the limit another engine needs.
int configureKernels(brt_engine* e) {
  static std::mutex mu;
  static std::map<int, uint32_t> highWater;
  std::lock_guard<std::mutex> lock(mu);
  uint32_t& mx = highWater[e->device];
  mx = std::max(mx, e->Mmax);
  BRT_CUDA_TRY(configureFusedKernels(mx));
  BRT_CUDA_TRY(configureFlockKernels(mx));
  BRT_CUDA_TRY(configureSchoolKernels(mx));
  return BRT_OK;
}
}  // namespace
