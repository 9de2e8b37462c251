// A user plugin written against the C++ facade: it keeps per-agent arrays of
// its own (DeviceArrayWrapper over Feature::User), which the engine moves with
// the agents at every reorder, and does its own device work in stream order
// through DeviceInterface::kernelCall.  The work here is a device-to-device
// copy of each agent's position into the plugin's array; after more steps the
// copy must still sit with the agent it was taken from.  Exits 0 on success.
#include <cuda_runtime.h>

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
  const float dt = 0.1f;
  engine.reset();

  // the reference's constructor form: a plugin array on the device interface
  DeviceArrayWrapper<uint32_t> tag(m_CommonRes.getDeviceInterface(), (int)n, 1, true, false);
  DeviceArrayWrapper<float4v> snapshot(Feature::User, (int)n);
  for (uint32_t i = 0; i < n; ++i) {
    const uint32_t v = 3u * i + 1u;
    tag.setHostArrayElement((int)i, &v);
  }
  tag.copyArrayToDevice();
  engine.step(dt, 3);

  // positions after 3 steps, by agent id
  engine.getPos()->copyArrayFromDevice();
  std::vector<float4v> pos3(engine.getPos()->getHostArray(), engine.getPos()->getHostArray() + n);

  // the plugin's own work: snapshot[slot] = pos[slot], on the engine stream
  bool before = false, after = false;
  m_CommonRes.getDeviceInterface()->kernelCall(
      [&](void* stream, const brt_arrays& a) {
        cudaMemcpyAsync(a.user[snapshot.getUserArrayId()], a.pos4, (size_t)a.num_agents * 16, cudaMemcpyDeviceToDevice,
                        (cudaStream_t)stream);
      },
      [&] { before = true; }, [&] { after = true; }, true);

  for (int f = 0; f < 4; ++f) {
    engine.reorderSimData();
    engine.computeNeighborhoods();
    engine.resetSteerForce();
    engine.computeSeparations();
    engine.computeAlignments();
    engine.computeCohesions();
    engine.computeSeekingsWorldCenter();
    engine.applySteeringForces(dt);
  }
  engine.step(dt, 5);

  tag.copyArrayFromDevice();
  snapshot.copyArrayFromDevice();
  // the wrappers' device arrays are the engine view's
  brt_arrays view;
  check(brt_engine_get_arrays(m_CommonRes.engine(), &view), "brt_engine_get_arrays");
  int field = -1;
  snapshot.bindToField(field);
  const bool arraysOk = snapshot.getReadDeviceArray() == (float4v*)view.user[snapshot.getUserArrayId()] &&
                        engine.getPos()->getWriteDeviceArray() == (float4v*)view.pos4 &&
                        engine.getPos()->getReadDeviceArray() == (float4v*)view.sorted_pos4 &&
                        field == (int)snapshot.getUserArrayId();
  std::printf("device arrays: %s\n", arraysOk ? "yes" : "no");
  // a plugin array holds one element per agent: other sizes are refused
  bool refused = false;
  try {
    DeviceArrayWrapper<uint32_t> bad(Feature::User, (int)n - 1);
  } catch (const std::runtime_error&) {
    refused = true;
  }
  std::printf("wrong size refused: %s\n", refused ? "yes" : "no");
  bool ok = before && after && arraysOk && refused;
  for (uint32_t i = 0; i < n && ok; ++i) ok = tag.getHostArray()[i] == 3u * i + 1u;
  const bool tagsOk = ok;
  ok = ok && std::memcmp(snapshot.getHostArray(), pos3.data(), n * sizeof(float4v)) == 0;
  std::printf("agents %u, tags follow their agents: %s, snapshot follows its agents: %s\n", n, tagsOk ? "yes" : "no",
              ok ? "yes" : "no");
  return ok ? 0 : 1;
}
