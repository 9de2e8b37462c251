// Reads a reference-style configuration into the facade's mixin engine
// without touching a GPU (the engine is created lazily) and prints the
// resulting parameters, so the configuration mapping can be checked on CPU.
#include <cstdio>

#include "behavert/BehaveRT.h"

using namespace BehaveRT;
typedef OpenSteerWrapperPlugIn<Proximity3DPlugIn<EnvGrid3DPlugIn<Body3DPlugIn<DummyPlugIn>>>> CrowdEngine;

int main(int argc, char** argv) {
  m_CommonRes.initialize(argc > 1 ? argv[1] : "");
  CrowdEngine engine;
  const brt_params& p = m_CommonRes.params();
  std::printf("numBodies %u worldSize %g cellSize %g maxBodiesPerCell %u maxNeighbors %u radius %g blockSize %d\n",
              p.numBodies, p.worldSize, p.cellSize, p.maxBodiesPerCell, p.maxNeighbors, p.commonSearchRadius,
              m_CommonRes.blockSize);
  return 0;
}
