// The BehaviorClustering plugin's interactive operations through the C++
// facade: calcInverseHash (agent id -> sorted slot) against getSortedIndex,
// and mergeClusters against a host restatement of the reference's merge
// kernel over the same labels and positions.  Exits 0 on success.
#include <cmath>
#include <cstdio>
#include <map>
#include <vector>

#include "behavert/BehaveRT.h"

using namespace BehaveRT;
typedef BehaviorClusteringPlugIn<OpenSteerWrapperPlugIn<Proximity3DPlugIn<EnvGrid3DPlugIn<Body3DPlugIn<DummyPlugIn>>>>>
    ClusterEngine;

int main(int argc, char** argv) {
  m_CommonRes.initialize(argc > 1 ? argv[1] : "");
  m_CommonRes.params().featuresCount = 4;
  ClusterEngine engine;
  const uint32_t n = m_CommonRes.params().numBodies;
  engine.reset();
  engine.reorderSimData();
  engine.computeNeighborhoods();
  engine.computeClusterMembership();

  // inverse hash: inverse[getSortedIndex(i)] == i for every sorted slot i
  engine.calcInverseHash();
  const std::vector<uint32_t>& inv = engine.getInverseHash();
  engine.getHash()->copyArrayFromDevice();
  bool invOk = inv.size() == n;
  for (uint32_t i = 0; i < n && invOk; ++i) invOk = inv[engine.getSortedIndex(i, false)] == i;

  // the two largest clusters' leaders
  const std::vector<float4v> member = engine.getClusterMembership();
  std::map<int, int> size;
  for (const float4v& m : member) ++size[(int)m.x];
  int a = -1, b = -1;
  for (const auto& kv : size) {
    if (a < 0 || kv.second > size[a]) { b = a; a = kv.first; }
    else if (b < 0 || kv.second > size[b]) b = kv.first;
  }
  engine.getPos()->copyArrayFromDevice();
  engine.getForward()->copyArrayFromDevice();
  std::vector<float4v> pos(engine.getPos()->getHostArray(), engine.getPos()->getHostArray() + n);
  std::vector<float4v> fwd0(engine.getForward()->getHostArray(), engine.getForward()->getHostArray() + n);
  engine.mergeClusters(a, b);
  engine.freezeClusters(a);
  engine.getForward()->copyArrayFromDevice();
  const float4v* fwd1 = engine.getForward()->getHostArray();
  const float4v pa = pos[engine.getSortedIndex((uint)a, false)], pb = pos[engine.getSortedIndex((uint)b, false)];
  const float speed = m_CommonRes.params().commonMaxSpeed;
  uint32_t moved = 0;
  bool mergeOk = a >= 0 && b >= 0 && a != b;
  for (uint32_t id = 0; id < n && mergeOk; ++id) {
    const int mine = (int)member[id].x;
    float4v want = fwd0[id];
    if (mine == a || mine == b) {
      const float4v& from = mine == a ? pa : pb;
      const float4v& to = mine == a ? pb : pa;
      const float dx = to.x - from.x, dy = to.y - from.y, dz = to.z - from.z;
      const float l = 1.0f / std::sqrt(dx * dx + dy * dy + dz * dz);
      want = float4v{dx * l, dy * l, dz * l, speed};
      ++moved;
    }
    mergeOk = want.x == fwd1[id].x && want.y == fwd1[id].y && want.z == fwd1[id].z && want.w == fwd1[id].w;
  }
  std::printf("agents %u, inverse hash: %s, merged %u agents of clusters %d and %d: %s\n", n, invOk ? "yes" : "no",
              moved, a, b, mergeOk ? "yes" : "no");
  return invOk && mergeOk && moved > 0 ? 0 : 1;
}
