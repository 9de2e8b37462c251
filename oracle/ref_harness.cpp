// ref_harness.cpp -- C entry points over the reference's own device
// functions, compiled on the host by oracle/build_ref.py (TEST
// INFRASTRUCTURE: the oracle is checked against these; nothing of the
// product links them).
//
// The included files are the reference's, where they lie; only the loops
// that the reference writes inside __global__ kernels (one agent's 27-cell
// visit, the flocking demo's steering sequence) are restated here, each
// citing its kernel.  The reference's grid is the clamped, non-periodic box
// with origin 0: callers use agents whose 27 cells lie inside the grid.
#include "common_resources.cu"
#include "../PlugIns/OpenSteerWrapper/OpenSteerWrapper_resources.cu"
#include "../PlugIns/Proximity3D/Proximity3D_kernel.cu"
#include "../PlugIns/OpenSteerWrapper/OpenSteerWrapper_kernel.cu"

// EnvGrid3D's texture hooks live in envgrid3d_kernel.cu, which is not built
// here (it is the reorder stage, with graphics interop): the plugin hooks of
// the files above call them, and the harness binds every texture itself.
extern "C" {
void EnvGrid3D::EnvGrid3D_beforeKernelCall() {}
void EnvGrid3D::EnvGrid3D_afterKernelCall() {}
}

#include <cstdint>

extern "C" {

// One flock's parameters, in the fields the reference's structs hold.
struct brt_ref_world {
  uint32_t gridSize;         // cells per side (EnvGrid3DParams.gridSize)
  float cellSize;            // EnvGrid3DParams.cellSize (world origin 0)
  uint32_t maxBodiesPerCell; // EnvGrid3DParams.maxBodiesPerCell (scan cap per cell)
  uint32_t maxNeighbors;     // Proximity3DParams.maxNeighbors
  uint32_t useKnn;           // Proximity3DParams.useKnn
  float searchRadius;        // Proximity3DParams.commonSearchRadius
  float maxSpeed, maxForce, mass, sensingMinRadius;  // OpenSteerWrapperParams
  float separation[3], alignment[3], cohesion[3];    // weight, radius, cosMaxAngle
};

// Binds the sorted arrays the reference reads through textures:
// cellStart (numCells words, 0xFFFFFFFF empty), agentHash (sorted (cell, id)
// pairs; n + maxBodiesPerCell entries, the tail holding a hash that matches
// no cell, as the reference's texture reads past the end return), sorted
// positions and forwards (float4; forward.w = speed).
int brt_ref_setup(const brt_ref_world* w, const uint32_t* cellStart, const uint32_t* agentHash, const float* posS,
                  const float* fwdS) {
  const uint32_t G = w->gridSize;
  dEnvGrid3DParams.gridSize = make_uint3(G, G, G);
  dEnvGrid3DParams.numCells = G * G * G;
  dEnvGrid3DParams.worldOrigin = make_float3(0.0f, 0.0f, 0.0f);
  dEnvGrid3DParams.cellSize = make_float3(w->cellSize, w->cellSize, w->cellSize);
  dEnvGrid3DParams.maxBodiesPerCell = w->maxBodiesPerCell;
  dProximity3DParams.useKnn = w->useKnn != 0;
  dProximity3DParams.maxNeighbors = w->maxNeighbors;
  dProximity3DParams.commonSearchRadius = w->searchRadius;
  dOpenSteerWrapperParams.commonMaxSpeed = w->maxSpeed;
  dOpenSteerWrapperParams.commonMaxForce = w->maxForce;
  dOpenSteerWrapperParams.commonMass = w->mass;
  dOpenSteerWrapperParams.commonSensingMinRadius = w->sensingMinRadius;
  dOpenSteerWrapperParams.separationParams = make_float3(w->separation[0], w->separation[1], w->separation[2]);
  dOpenSteerWrapperParams.alignmentParams = make_float3(w->alignment[0], w->alignment[1], w->alignment[2]);
  dOpenSteerWrapperParams.cohesionParams = make_float3(w->cohesion[0], w->cohesion[1], w->cohesion[2]);
  dBody3DParams.use2DProjection = false;
  cellStartTex.data = cellStart;
  agentHashTex.data = reinterpret_cast<const uint2*>(agentHash);
  oldPosTex.data = reinterpret_cast<const float4*>(posS);
  oldForwardTex.data = reinterpret_cast<const float4*>(fwdS);
  return 0;
}

// The neighbour list of sorted slot `index`: genericCalcNeighgborhoodD's
// loop (PlugIns/Proximity3D/Proximity3D_kernel.cu:89-125), x outer, z inner,
// over checkForNeighborsInCell (Proximity3D_resources.cu:111-172).
int brt_ref_neighbors(uint32_t index, uint32_t* list, uint32_t* count) {
  const float4 pos = FETCH(oldPos, index);
  const int3 gridPos = calcGridPos(pos, dEnvGrid3DParams.worldOrigin, dEnvGrid3DParams.cellSize);
  uint neighNum = 0;
  uint neighList[Proximity3d_MAX_NEIGHBORS];
  float distList[Proximity3d_MAX_NEIGHBORS];
  float maxDistValue = 0;
  for (int x = -1; x <= 1; x++)
    for (int y = -1; y <= 1; y++)
      for (int z = -1; z <= 1; z++)
        Proximity3D::checkForNeighborsInCell(gridPos + make_int3(x, y, z), index, pos, neighNum, neighList, distList,
                                             maxDistValue);
  for (uint k = 0; k < neighNum; ++k) list[k] = neighList[k];
  *count = neighNum;
  return 0;
}

// The flocking demo's steering force of sorted slot `index` from its list:
// resetSteerForce, then genericSeparationD, genericAlignmentD and
// genericCohesionD (OpenSteerWrapper_kernel.cu:62-178, in the order of
// BehaveRT_Flocking.cpp:183-190), each adding weight * calcX to the force
// through storeSteeringForce<true> (OpenSteerWrapper_resources.cu:113-124).
int brt_ref_steer(uint32_t index, const uint32_t* list, uint32_t count, float* steer3) {
  const float3 myPos = make_float3(tex1Dfetch(oldPosTex, index));
  const float3 myForward = make_float3(tex1Dfetch(oldForwardTex, index));
  uint neighList[Proximity3d_MAX_NEIGHBORS];
  for (uint k = 0; k < count; ++k) neighList[k] = list[k];
  float3 force = make_float3(0.0f, 0.0f, 0.0f);
  float3 s = OpenSteerWrapper::calcSeparation(myPos, myForward, count, neighList) *
             dOpenSteerWrapperParams.separationParams.x;
  s += force;
  force = s;
  float3 a = OpenSteerWrapper::calcAlignment(myPos, myForward, count, neighList) *
             dOpenSteerWrapperParams.alignmentParams.x;
  a += force;
  force = a;
  float3 c = OpenSteerWrapper::calcCohesion(myPos, myForward, count, neighList) *
             dOpenSteerWrapperParams.cohesionParams.x;
  c += force;
  force = c;
  steer3[0] = force.x; steer3[1] = force.y; steer3[2] = force.z;
  return 0;
}

// applySteeringForceSingle (OpenSteerWrapper_resources.cu:326-379) on one
// agent: in/out speed, forward (xyz), position (xyz), smoothed acceleration.
int brt_ref_integrate(const float* force3, float elapsedTime, float* speed, float* forward3, float* position3,
                      float* smoothedAccel3) {
  float3 forward = make_float3(forward3[0], forward3[1], forward3[2]);
  float3 position = make_float3(position3[0], position3[1], position3[2]);
  float3 acc = make_float3(smoothedAccel3[0], smoothedAccel3[1], smoothedAccel3[2]);
  OpenSteerWrapper::applySteeringForceSingle(make_float3(force3[0], force3[1], force3[2]), elapsedTime,
                                             dOpenSteerWrapperParams.commonMaxForce,
                                             dOpenSteerWrapperParams.commonMaxSpeed,
                                             dOpenSteerWrapperParams.commonMass, *speed, forward, position, acc);
  forward3[0] = forward.x; forward3[1] = forward.y; forward3[2] = forward.z;
  position3[0] = position.x; position3[1] = position.y; position3[2] = position.z;
  smoothedAccel3[0] = acc.x; smoothedAccel3[1] = acc.y; smoothedAccel3[2] = acc.z;
  return 0;
}

// adjustRawSteeringForce (Core/common_resources.cu:234-254) alone.
int brt_ref_adjust(const float* force3, float speed, const float* forward3, float maxSpeed, float* out3) {
  const float3 r = adjustRawSteeringForce(make_float3(force3[0], force3[1], force3[2]), speed,
                                          make_float3(forward3[0], forward3[1], forward3[2]), maxSpeed);
  out3[0] = r.x; out3[1] = r.y; out3[2] = r.z;
  return 0;
}

// calcGridHash(calcGridPos(p)) (envgrid3d_resources.cu:60-84).
uint32_t brt_ref_hash(const float* pos4) {
  const float4 p = make_float4(pos4[0], pos4[1], pos4[2], pos4[3]);
  return calcGridHash(calcGridPos(p, dEnvGrid3DParams.worldOrigin, dEnvGrid3DParams.cellSize),
                      dEnvGrid3DParams.gridSize);
}

// One frame of the flocking demo (BehaveRT_Flocking.cpp:180-196) through the
// reference's own kernels, each run on the host thread by thread
// (blockDim = 1, blockIdx.x = the agent's sorted slot):
//   genericCalcNeighgborhoodD  (Proximity3D_kernel.cu:89-125)
//   resetSteerForce, then genericSeparationD, genericAlignmentD,
//   genericCohesionD            (OpenSteerWrapper_kernel.cu:62-178), each
//                               reading the previous force and writing the
//                               next (the double-buffered steerForce feature)
//   genericApplySteeringForceD (OpenSteerWrapper_kernel.cu:265-333)
// The sort, reorder and cellStart stages are inputs: agentHash holds the
// sorted (cell, id) pairs (padded as for brt_ref_setup), posS / fwdS / accS
// the sorted state, cellStart the first sorted slot of each cell.  Outputs:
// lists (n * (maxNeighbors + 1) words, per sorted slot, as the reference
// writes them) and the new state by agent id (float4 each).  The reference
// reads the lists back in uint4 words, 4 * (maxNeighbors / 4 + 1) to an
// agent (Proximity3DPlugIn.h:148-149), which is the writer's stride only
// when maxNeighbors % 4 == 3; callers use such sizes.
int brt_ref_frame(uint32_t n, float elapsedTime, const uint32_t* cellStart, const uint32_t* agentHash,
                  const float* posS, const float* fwdS, const float* accS, uint32_t* lists, float* pos_out,
                  float* fwd_out, float* acc_out) {
  enum { kPos, kHash, kCellStart, kNeighList, kForward, kAccel, kForce };
  dBody3DFields.position = kPos;
  dEnvGrid3DFields.hash = kHash;
  dProximity3DFields.cellStart = kCellStart;
  dProximity3DFields.neighList = kNeighList;
  dOpenSteerWrapperFields.forward = kForward;
  dOpenSteerWrapperFields.smoothAccel = kAccel;
  dOpenSteerWrapperFields.steerForce = kForce;
  dOpenSteerWrapperDynParams.elapsedTime = elapsedTime;
  dProximity3DParams.numNeighWordsPerAgent = dProximity3DParams.maxNeighbors / 4 + 1;
  cellStartTex.data = cellStart;
  agentHashTex.data = reinterpret_cast<const uint2*>(agentHash);
  oldPosTex.data = reinterpret_cast<const float4*>(posS);
  oldForwardTex.data = reinterpret_cast<const float4*>(fwdS);
  oldSmoothedAccelTex.data = reinterpret_cast<const float4*>(accS);
  auto forAll = [n](void (*kernel)()) {
    for (uint32_t i = 0; i < n; ++i) {
      blockIdx.x = i;
      kernel();
    }
  };
  deviceDataRepository[kNeighList].outputDataPointer = lists;
  forAll(&genericCalcNeighgborhoodD);
  oldNeighListTex.data = reinterpret_cast<const uint4*>(lists);
  float4* force[2] = {new float4[n](), new float4[n]()};  // resetSteerForce: zero
  void (*behaviours[3])() = {&genericSeparationD, &genericAlignmentD, &genericCohesionD};
  int cur = 0;
  for (auto k : behaviours) {
    oldForceTex.data = force[cur];
    deviceDataRepository[kForce].outputDataPointer = force[cur ^ 1];
    forAll(k);
    cur ^= 1;
  }
  oldForceTex.data = force[cur];
  deviceDataRepository[kPos].outputDataPointer = pos_out;
  deviceDataRepository[kForward].outputDataPointer = fwd_out;
  deviceDataRepository[kAccel].outputDataPointer = acc_out;
  forAll(&genericApplySteeringForceD);
  delete[] force[0];
  delete[] force[1];
  blockIdx.x = 0;
  return 0;
}

}  // extern "C"
