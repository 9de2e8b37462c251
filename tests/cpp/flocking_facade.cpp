// The reference's flocking application shape, compiled against the C++
// facade: a mixin engine configured from a [Section] key = value file, run
// stage by stage (BehaveRT_Flocking.cpp:177-199) and then with the fused
// step from the same reset state.  Exits 0 when both give identical states.
#include <cstdio>
#include <cstring>
#include <vector>

#include "behavert/BehaveRT.h"

using namespace BehaveRT;
typedef OpenSteerWrapperPlugIn<Proximity3DPlugIn<EnvGrid3DPlugIn<Body3DPlugIn<DummyPlugIn>>>> CrowdEngine;

int main(int argc, char** argv) {
  m_CommonRes.initialize(argc > 1 ? argv[1] : "");
  CrowdEngine engine;
  const uint32_t n = m_CommonRes.params().numBodies;
  const int frames = 5;
  const float dt = 0.1f;

  engine.reset();
  for (int f = 0; f < frames; ++f) {
    engine.reorderSimData();
    engine.computeNeighborhoods();
    engine.resetSteerForce();
    engine.computeSeparations();
    engine.computeAlignments();
    engine.computeCohesions();
    engine.computeSeekingsWorldCenter();
    engine.applySteeringForces(dt);
  }
  engine.getPos()->copyArrayFromDevice();
  engine.getForward()->copyArrayFromDevice();
  std::vector<float4v> posA(engine.getPos()->getHostArray(), engine.getPos()->getHostArray() + n);
  std::vector<float4v> fwdA(engine.getForward()->getHostArray(), engine.getForward()->getHostArray() + n);

  engine.reset();
  engine.step(dt, frames);
  engine.getPos()->copyArrayFromDevice();
  engine.getForward()->copyArrayFromDevice();
  const bool same = std::memcmp(posA.data(), engine.getPos()->getHostArray(), n * sizeof(float4v)) == 0 &&
                    std::memcmp(fwdA.data(), engine.getForward()->getHostArray(), n * sizeof(float4v)) == 0;
  const uint sorted0 = engine.getSortedIndex(0);
  std::printf("agents %u, frames %d, stage-wise == fused: %s, agent at sorted slot 0: %u\n", n, frames,
              same ? "yes" : "no", sorted0);
  return same ? 0 : 1;
}
