// brt_kernels.cuh -- argument blocks and launchers of the pipeline kernels.
#pragma once

#include "brt_internal.cuh"

namespace brt {

constexpr uint32_t kFusedThreads = 128;
constexpr uint32_t kFlockMaxThreads = 256;  // largest block of the single-pass flock kernel

struct HashArgs {
  const float4* pos;           // canonical slot order
  const uint32_t* id;          // agent id per canonical slot
  uint2* pairs;                // out, agent-id order: (key, slot)
  const FlockDev* flocks;
  const uint32_t* agentBase;   // nflocks + 1
  uint32_t nflocks, n;
  uint32_t passes, bins;
  uint32_t shift[4], mask[4];
  uint32_t* hist;              // passes * bins, accumulated with atomics
  uint32_t* cellStart;
  uint32_t* cellEnd;
  uint32_t cellWords4;         // cell words / 4 (arrays padded to 4)
  uint32_t* status;            // sort look-back state to clear
  uint32_t statusWords;
  uint32_t* counters;          // sort tile counters to clear
  uint32_t* stepCounter;       // random-stream step counter, incremented once per step
  const uint32_t* gate;        // optional: run only when *gate == kResortFullSort
  uint32_t* resortValid;       // optional: cleared (the cell ranges are cleared here)
};

struct ReorderArgs {
  const uint2* pairs;          // sorted (key, previous slot)
  const float4* posA; const float4* fwdA; const float4* accA;
  const float* featA; const uint32_t* idA;
  float4* posS; float4* fwdS; float4* accS; float* featS; uint32_t* idS;
  uint32_t* prevOut;           // source slot per sorted slot (optional, adjoint tape)
  uint32_t fs4;                // feature float4s per agent
  uint32_t* cellStart; uint32_t* cellEnd;
  uint32_t* hist; uint32_t histWords;
  uint32_t n, numCells;
  uint32_t* errWord;
  // incremental re-sort (all null outside the fused step)
  const uint32_t* resortMode;  // the step's sort mode
  const uint32_t* newStart;    // per cell, from the re-sort's cell scan
  uint32_t* moverCount; uint32_t* moverHead;  // reset for every cell seen
  uint32_t* resortValid;       // set: the next step may re-sort from this order
  // cell-cull gate of scan variants 0 and 1 (null: not computed).  Words
  // [0] and [1] are the launch's accumulator and block ticket, both back at
  // zero when the launch ends; [2] is set to nonzero when a sorted position
  // is NaN or outside [0, L] on some axis of its flock's world.
  uint32_t* cullWords;
  const FlockDev* flocks; const uint32_t* agentBase; uint32_t nflocks;
};

struct FusedArgs {
  const float4* posS; const float4* fwdS; const float4* accS;
  const float* featS; const uint32_t* idS;
  float4* posA; float4* fwdA; float4* accA; float* featA; uint32_t* idA;
  float4* statsById;
  const uint32_t* cellStart; const uint32_t* cellEnd;
  const FlockDev* flocks; const uint32_t* agentBase;
  const float4* obstacles;
  const uint2* obsMask;          // per-cell obstacle field (global cell index) or null
  uint32_t* lists;             // optional, stride listStride
  uint32_t listStride;
  uint32_t nflocks, n, Mmax, Fs;
  float dt;
  int scanVariant;             // 0: pipelined x4 + cell culling, 1: x2 + culling, 2: x4, 3: flat loop,
                               // 4: warp-cooperative, 5: warp-cooperative with windows,
                               // 6: staged tiles (tileFlockKernel), 7: warp-cooperative with
                               // bounding-box culling
  const uint32_t* stepCounter; // random-stream step of the Schooling move
  const uint32_t* cullGate;    // scan variants 0 and 1: cells are culled only when
                               // this word is zero (null: never culled)
  // scan variant 6: the (flock, row segment) tiles and the work-queue counter
  const uint4* tiles;          // x flock, y row y | z << 16, z first x | cells << 16
  uint32_t numTiles;
  uint32_t* tileCounter;       // zeroed before each launch
  uint32_t tileBlocks;         // persistent blocks of the launch
};
// Home cells per tile (one row segment) and staged candidates per tile.
constexpr uint32_t kTileMaxCells = 32;
constexpr uint32_t kTileThreads = 128;

struct StageArgs {
  const float4* posS; const float4* fwdS; const float4* accS;
  const float* featS; const uint32_t* idS;
  float4* posA; float4* fwdA; float4* accA; float* featA; uint32_t* idA;
  float4* statsById;
  float4* steer;
  float4* fwdW;                  // the sorted forwards again, written by the avoid-neighbours stage
  float avoidBase[3];            // move-away stage: the point to flee
  float avoidBaseParams[3];      //   (steering weight, acceleration factor, radius)
  const uint32_t* cellStart; const uint32_t* cellEnd;
  const FlockDev* flocks; const uint32_t* agentBase;
  const float4* obstacles;
  const uint2* obsMask;          // per-cell obstacle field (global cell index) or null
  uint32_t* lists;
  uint32_t listStride;
  uint32_t nflocks, n, Fs;
  const uint32_t* stepCounter;
};

// Incremental re-sort (brt_resort.cu).  words[]: mode of the current step,
// previous order valid (set by the fused step's reorder, cleared by the hash
// kernel and by the host whenever the canonical order may have changed),
// movers counted, a cell's mover list overflowed.
constexpr uint32_t kResortChunk = 1024;   // slots per stayer-count block
constexpr uint32_t kMaxMoversPerCell = 32;
constexpr uint32_t kNoMover = 0xFFFFFFFFu;
constexpr uint32_t kResortWordMode = 0, kResortWordValid = 1, kResortWordMovers = 2, kResortWordOverflow = 3;
constexpr uint32_t kResortWordDone = 4;  // blocks of the mark kernel finished
constexpr uint32_t kResortWords = 8;
struct ResortArgs {
  const float4* pos;             // canonical positions (previous sorted order)
  const uint32_t* id;            // agent id per canonical slot
  const uint2* prevPairs;        // previous step's sorted pairs: the previous key of each slot
  const uint32_t* cellStart; const uint32_t* cellEnd;  // previous step's cell ranges
  const FlockDev* flocks; const uint32_t* agentBase;
  uint32_t nflocks, n, numCells;
  uint32_t maxMovers;            // the full sort runs above this many movers
  uint32_t* newKey;              // [n]
  uint32_t* prefix;              // [n] stayers before the slot in its block, stay flag in bit 31
  uint32_t* blockStay;           // [blocks + 1] stayer counts, then their exclusive scan
  uint32_t* moverCount;          // [numCells], zero between steps
  uint32_t* moverHead;           // [numCells], kNoMover between steps
  uint32_t* moverNext;           // [n]
  uint32_t* newStart;            // [numCells] first sorted position of each cell
  uint32_t* stayBase;            // [numCells] newStart minus the stayers before the cell's previous range
  uint32_t* tileStatus;          // [cell tiles] look-back state of the cell scan
  uint32_t* tileCounter;
  uint32_t* words;               // [kResortWords]
  uint32_t* stepCounter;         // random-stream step (advanced here when the hash does not run)
  uint2* out;                    // sorted pairs: the sort's final buffer
  uint32_t* errWord;
  LookbackWait wait;             // bound of the cell scan's look-back
};
uint32_t resortBlocks(uint32_t n);
uint32_t resortCellTiles(uint32_t numCells);
cudaError_t launchResortMark(const ResortArgs& A, cudaStream_t st);
cudaError_t launchResortPlace(const ResortArgs& A, cudaStream_t st);

// Reverse of one taped step (brt_adjoint.cu).
constexpr uint32_t kAdjointThreads = 128;
struct AdjointStepArgs {
  const float4* posS; const float4* fwdS; const float4* accS;   // the step's sorted input state
  const uint32_t* lists; uint32_t listStride;                    // its neighbour lists (sorted slots)
  const uint32_t* prev;                                          // canonical slot of each sorted slot
  const uint32_t* idS;                                           // agent id per sorted slot
  const FlockDev* flocks; const uint32_t* agentBase; const float4* obstacles;
  const uint2* obsMask;
  uint32_t nflocks, n;
  float dt;
  const float4* gOutP; const float4* gOutF; const float4* gOutA; // output adjoint by sorted slot
  float4* gInP; float4* gInF; float4* gInA;                      // input adjoint by canonical slot
  // Emit -> gather hand-over of one step (sorted slots of this step):
  float4* contrib;      // 2 per list entry e = i * entryStride + k, for in-list overflow only: the
                        // position adjoint (xyz) and forward adjoint (w, then xy) agent i sends
                        // the agent it lists at k
  float4* selfP;        // per slot: the agent's own position adjoint terms
  float4* selfF;        // per slot: the agent's own forward adjoint terms (w: speed)
  // In-lists (the transposed neighbour list of the step): the contribution
  // of entry e = i * entryStride + k (agent i lists j at position k) goes to
  // inbox[2 * (j * inCap + q)] (two float4) at q = atomicAdd(&inCount[j], 1);
  // entries beyond inCap go to contrib[2 * e] and a linked overflow list
  // (ovHead[j], ovNext[e]).  The gather resets inCount and ovHead for the
  // next-earlier step.
  uint32_t* inCount; float4* inbox; uint32_t inCap;
  uint32_t* ovHead; uint32_t* ovNext;
  uint32_t entryStride; // list positions per slot in the entry code (maxNeighbors, <= 32)
  double* accW;         // per agent id: the weight adjoint summed over the steps (3 doubles)
  uint32_t* exportLists;                                         // optional, by agent id
  uint32_t* exportFlags;                                         // optional, 4 words by agent id
  float4* exportState;                                           // optional: pos, fwd, acc by agent id
};
constexpr uint32_t kNoEntry = 0xFFFFFFFFu;
// Per-flock FP64 sums of per-item values (the weight adjoint, the loss), in
// a fixed order: kReduceParts blocks per flock, each over a fixed part of the
// flock's items, then the parts in order.
constexpr uint32_t kReduceParts = 32;
struct FlockReduceArgs {
  const double* vals; uint32_t width;   // width (1..3) doubles per item
  const uint32_t* agentBase;            // items of flock f: [agentBase[f], agentBase[f+1])
  uint32_t nflocks;
  double* partial;                      // nflocks * kReduceParts * width scratch
  double* out;                          // nflocks * width, written
};
struct LossArgs {
  const float4* posA; const uint32_t* idA;    // final state, canonical order
  const float4* target;                       // by agent id
  const FlockDev* flocks; const uint32_t* agentBase;
  uint32_t nflocks, n;
  double* lossTerm;                           // per canonical slot (reduced per flock afterwards)
  float4* gT;                                 // unscaled terminal position adjoint, canonical order
};
struct SeedArgs {
  const float4* gT; const float* scale;       // scale per flock (device) or null for 1
  const float4* extraP; const float4* extraF; const float4* extraA;  // optional, by agent id
  const uint32_t* idA;
  const uint32_t* agentBase;
  uint32_t nflocks, n;
  float4* gP; float4* gF; float4* gA;
};
struct OutArgs {
  const float4* gP; const float4* gF; const float4* gA;
  const uint32_t* id0; const float4* fwd0;    // initial canonical order
  uint32_t n;
  float4* outP; float4* outF; float4* outA; float4* outV;  // by agent id, each optional
};
cudaError_t launchAdjointStep(const AdjointStepArgs& A, cudaStream_t st);
cudaError_t launchFlockReduce(const FlockReduceArgs& A, cudaStream_t st);
cudaError_t launchLoss(const LossArgs& A, cudaStream_t st);
cudaError_t launchAdjointSeed(const SeedArgs& A, cudaStream_t st);
cudaError_t launchAdjointOut(const OutArgs& A, cudaStream_t st);

cudaError_t launchHash(const HashArgs& A, uint32_t maxBlocks, cudaStream_t st);
cudaError_t launchReorder(const ReorderArgs& A, cudaStream_t st);
cudaError_t launchFused(const FusedArgs& A, bool knn, cudaStream_t st);
cudaError_t launchFlock(const FusedArgs& A, int phase2, uint32_t block, int regs, cudaStream_t st);
uint32_t tileFlockBlocks(uint32_t Mmax, uint32_t Fs, int smCount);
cudaError_t launchLists(const StageArgs& A, bool knn, cudaStream_t st);
cudaError_t launchSteerStage(const StageArgs& A, int which, cudaStream_t st);
cudaError_t launchIntegrateStage(const StageArgs& A, float dt, cudaStream_t st);
// Schooling (brt_school.cu): fused step, and stage which = 0 repulsion,
// 1 attraction/orientation, 2 move, 3 animateSchool.
cudaError_t launchSchool(const FusedArgs& A, cudaStream_t st);
cudaError_t launchSchoolStage(const StageArgs& A, int which, cudaStream_t st);
cudaError_t configureSchoolKernels(uint32_t Mmax);
// BehaviorClustering analytics (brt_cluster.cu): which = 0 reset labels,
// 1 one propagation sweep, 2 hit rate; in / out are the membership buffers.
struct ClusterArgs {
  const float4* posS; const uint32_t* idS;
  const uint32_t* lists; uint32_t listStride;
  const FlockDev* flocks; const uint32_t* agentBase;
  uint32_t nflocks, n;
  float radius;
  const float4* in; float4* out;
};
cudaError_t launchCluster(const ClusterArgs& A, int which, cudaStream_t st);
cudaError_t launchScatterToId(const float4* src, const uint32_t* id, float4* dst, uint32_t n, cudaStream_t st);
cudaError_t launchScatterFeatToId(const float* src, uint32_t Fs, const uint32_t* id, float* dst, uint32_t F, uint32_t n, cudaStream_t st);
cudaError_t launchLoadFeat(const float* src, uint32_t F, float* dst, uint32_t Fs, uint32_t n, cudaStream_t st);
cudaError_t launchGatherFromId(const float4* src, const uint32_t* id, float4* dst, uint32_t n, bool forceW1, cudaStream_t st);
cudaError_t configureFusedKernels(uint32_t Mmax);
cudaError_t configureFlockKernels(uint32_t Mmax);
cudaError_t launchGatherFeatFromId(const float* src, uint32_t F, const uint32_t* id, float* dst, uint32_t Fs, uint32_t n, cudaStream_t st);
cudaError_t launchHashPairsOut(const uint2* pairs, const uint32_t* idS, uint32_t* keys, uint32_t* ids, uint32_t n, cudaStream_t st);
// dst[i] = src[index[i * stride]] and dst[index[i]] = src[i] for arrays of
// `words` 32-bit words per agent.
cudaError_t launchGatherWords(const uint32_t* src, const uint32_t* index, uint32_t stride, uint32_t* dst, uint32_t words,
                              uint32_t n, cudaStream_t st);
cudaError_t launchScatterWords(const uint32_t* src, const uint32_t* index, uint32_t* dst, uint32_t words, uint32_t n,
                               cudaStream_t st);

uint32_t sortPassMask(const SortPlan& p, uint32_t pass);

}  // namespace brt
