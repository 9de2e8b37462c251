// The reference's schooling application shape, compiled against the C++
// facade: the split Schooling functionalities (calcRepulsion ->
// calcAttractionOrientation -> calcMovement, SchoolingPlugIn.h:236-299) run
// frame by frame, then the fused step from the same reset state.  Exits 0
// when both give identical states.
#include <cstdio>
#include <cstring>
#include <vector>

#include "behavert/BehaveRT.h"

using namespace BehaveRT;
typedef SchoolingPlugIn<OpenSteerWrapperPlugIn<Proximity3DPlugIn<EnvGrid3DPlugIn<Body3DPlugIn<DummyPlugIn>>>>> SchoolEngine;

int main(int argc, char** argv) {
  m_CommonRes.initialize(argc > 1 ? argv[1] : "");
  SchoolEngine engine;
  const uint32_t n = m_CommonRes.params().numBodies;
  const int frames = 5;
  const float dt = 0.1f;

  engine.reset();
  for (int f = 0; f < frames; ++f) {
    engine.reorderSimData();
    engine.computeNeighborhoods();
    engine.calcRepulsion();
    engine.calcAttractionOrientation();
    engine.calcMovement();
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
  std::printf("agents %u, frames %d, speed %.2f, stage-wise == fused: %s\n", n, frames,
              engine.getForward()->getHostArray()[0].w, same ? "yes" : "no");
  return same ? 0 : 1;
}
