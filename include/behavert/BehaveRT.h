// BehaveRT.h -- header-only C++ facade of the reference's plugin engine over
// the C-ABI of libbehavert_b200.so.
//
// Keeps the reference's class names, mixin structure and per-frame method
// names so that an application written against the reference compiles
// against this header:
//   CommonResources m_CommonRes                      Core/include/CommonResources.h:62-126
//   DeviceInterface                                  Core/include/DeviceInterface.cuh:53-297
//   DeviceArrayWrapper<T>                            Core/include/DeviceArrayWrapper.h:58-192
//   SimEnginePlugIn / DummyPlugIn                    Core/include/SimEnginePlugIn.h:79-200
//   Body3DPlugIn / EnvGrid3DPlugIn / Proximity3DPlugIn / OpenSteerWrapperPlugIn /
//   BehaviorClusteringPlugIn                         PlugIns/*/include/*PlugIn.h
//   UtilityConfigFile ([Section] key = value)        Core/include/UtilityConfigFile.h:54-81
//
// Differences: there is no GL/VBO interop (arrays are plain device memory
// inside the engine), the world is the periodic cube [0, worldSize)^3, errors
// throw BehaveRT::Error instead of exiting, and the random initialisation of
// reset() uses an explicit seed instead of rand().
#pragma once

#include <algorithm>
#include <cstdarg>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <functional>
#include <map>
#include <list>
#include <memory>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../behavert_b200.h"

namespace BehaveRT {

typedef unsigned int uint;
typedef std::vector<std::string> DependenciesList;

struct float4v { float x, y, z, w; };
struct uint2v { uint32_t x, y; };

class Error : public std::runtime_error {
 public:
  Error(const std::string& where, int status)
      : std::runtime_error(where + ": " + brt_error_string(status) + " (" + brt_last_error() + ")"), status(status) {}
  int status;
};

inline void check(int status, const char* where) {
  if (status != BRT_OK) throw Error(where, status);
}

// ---------------------------------------------------------------------------
// [Section] key = value configuration (UtilityConfigFile).
class UtilityConfigFile {
 public:
  void load(const std::string& path) {
    std::ifstream in(path);
    if (!in) throw std::runtime_error("cannot open config file " + path);
    std::string line, section;
    while (std::getline(in, line)) {
      const size_t hash = line.find_first_of("#;");
      if (hash != std::string::npos) line = line.substr(0, hash);
      line = trim(line);
      if (line.empty()) continue;
      if (line.front() == '[' && line.back() == ']') { section = trim(line.substr(1, line.size() - 2)); continue; }
      const size_t eq = line.find('=');
      if (eq == std::string::npos) continue;
      m_Settings[section][trim(line.substr(0, eq))] = trim(line.substr(eq + 1));
    }
  }
  void setSetting(const std::string& key, const std::string& section, const std::string& value) {
    m_Settings[section][key] = value;
  }
  std::string getSetting(const std::string& key, const std::string& section, const std::string& def = "") const {
    auto s = m_Settings.find(section);
    if (s == m_Settings.end()) return def;
    auto k = s->second.find(key);
    return k == s->second.end() ? def : k->second;
  }
  bool has(const std::string& key, const std::string& section) const { return !getSetting(key, section).empty(); }

 private:
  static std::string trim(const std::string& s) {
    const size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
  }
  std::map<std::string, std::map<std::string, std::string>> m_Settings;
};

inline float parseFloat(const std::string& s) { return std::stof(s); }
inline int parseInt(const std::string& s) { return std::stoi(s); }
inline bool parseBool(const std::string& s) { return s == "true" || s == "1" || s == "yes"; }
inline void parseFloat3(const std::string& s, float* v) {
  std::istringstream in(s);
  in >> v[0] >> v[1] >> v[2];
}

// ---------------------------------------------------------------------------
// DeviceInterface: device selection, synchronisation and the engine handle.
class DeviceInterface {
 public:
  explicit DeviceInterface(int device = 0) : m_Device(device) {}
  ~DeviceInterface() { release(); }
  int device() const { return m_Device; }
  brt_engine* engine() const { return m_Engine; }
  bool hasEngine() const { return m_Engine != nullptr; }
  void createEngine(const brt_params& p) {
    release();
    check(brt_engine_create(&p, 1, m_Device, &m_Engine), "brt_engine_create");
  }
  void release() {
    if (m_Engine) brt_engine_destroy(m_Engine);
    m_Engine = nullptr;
  }
  // Core/DeviceInterface.cu:114-118
  void threadSync() {
    if (m_Engine) check(brt_sync(m_Engine), "brt_sync");
  }
  // kernelCall (Core/DeviceInterface.cu:380-458): the before hook, the
  // caller's launches on the engine stream over the engine's arrays, the
  // after hook, and an optional synchronisation.  `launch` receives the
  // stream (a cudaStream_t) and the brt_arrays view.
  using Launch = std::function<void(void* stream, const brt_arrays& arrays)>;
  void kernelCall(const Launch& launch, const std::function<void()>& before = {},
                  const std::function<void()>& after = {}, bool sync = false) {
    if (!m_Engine) throw std::runtime_error("kernelCall before the engine exists");
    if (before) before();
    struct Ctx { const Launch* fn; } ctx{&launch};
    check(brt_engine_launch(
              m_Engine, [](void* u, void* s, const brt_arrays* a) { (*static_cast<Ctx*>(u)->fn)(s, *a); }, &ctx),
          "kernelCall");
    if (after) after();
    if (sync) threadSync();
  }

 private:
  int m_Device;
  brt_engine* m_Engine = nullptr;
};

// ---------------------------------------------------------------------------
// UtilityLogger (Core/include/UtilityLogger.h:50-133): the last maxSize
// messages of (sender, text, level), each also written to standard output as
// "sender>> text"; a sender filter and a level (debug or info) select what a
// display shows.  quickLog formats printf-style.
class UtilityLogger {
 public:
  enum mLogLevels { LOG_DEBUG, LOG_INFO };
  typedef std::string msgSenderType;
  typedef std::string msgTextType;
  typedef std::pair<msgSenderType, msgTextType> logMsg;
  typedef std::pair<logMsg, mLogLevels> logItem;
  typedef std::list<logItem> msgListType;

  explicit UtilityLogger(unsigned int maxSize) : mMaxSize(maxSize) {}
  void log(msgSenderType msgSender, msgTextType msgText, mLogLevels level = LOG_INFO) {
    std::printf("%s>> %s\n", msgSender.c_str(), msgText.c_str());
    mMsgList.push_back(logItem(logMsg(msgSender, msgText), level));
    while (mMsgList.size() > mMaxSize) mMsgList.pop_front();
    mModified = true;
  }
  void quickLog(msgSenderType msgSender, const char* fmt, ...) {
    char msg[1024];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(msg, sizeof(msg), fmt, ap);
    va_end(ap);
    log(msgSender, msg);
  }
  bool checkSender(const logItem& item) const { return item.first.first == mSenderFilter; }
  bool checkLevel(const logItem& item) const { return item.second == mLevel || item.second == LOG_INFO; }
  std::string getMsgString(const logItem& item) const { return item.first.second; }
  void setLevelString(const std::string& level) { mLevel = level == "debug" ? LOG_DEBUG : LOG_INFO; }
  // the messages the level admits, oldest first, joined by `separator`
  std::string getMsgListString(const std::string& separator) const {
    std::string out;
    for (const logItem& item : mMsgList)
      if (checkLevel(item)) out += getMsgString(item) + separator;
    return out;
  }
  msgListType getMsgList() const { return mMsgList; }
  bool isModified() const { return mModified; }
  void setModified(bool modified) { mModified = modified; }
  void setSenderFilter(const std::string& senderFilter) { mSenderFilter = senderFilter; }
  std::string getSenderFilter() const { return mSenderFilter; }

  msgListType mMsgList;

 protected:
  unsigned int mMaxSize;
  mLogLevels mLevel = LOG_INFO;
  bool mModified = false;
  std::string mSenderFilter;
};

// ---------------------------------------------------------------------------
// CommonResources: configuration, device interface and the parameters the
// installed plugins fill in (the reference's hXParams globals).
class CommonResources {
 public:
  CommonResources() { brt_params_default(&m_Params); }
  void initialize(const std::string& configFileName) {
    if (!configFileName.empty()) m_Config.load(configFileName);
    m_Initialized = true;
  }
  bool isInitialized() const { return m_Initialized; }
  DeviceInterface* getDeviceInterface() { return &m_DeviceInterface; }
  UtilityConfigFile* getConfig() { return &m_Config; }
  // the reference keeps the last 50 messages (Core/src/CommonResources.cpp:58)
  UtilityLogger* getLogger() { return &m_Logger; }
  brt_params& params() { return m_Params; }
  // The engine is created the first time a functionality needs it, once
  // every plugin has installed its parameters.
  brt_engine* engine() {
    if (!m_DeviceInterface.hasEngine()) {
      m_DeviceInterface.createEngine(m_Params);
      // a configured block size that the flock kernel accepts (a multiple of
      // 32 up to 256); others leave the engine's default, with a message
      if (blockSize > 0) {
        if (blockSize % 32 == 0 && blockSize <= 256)
          check(brt_engine_set_option(m_DeviceInterface.engine(), "block_size", blockSize), "block_size");
        else
          m_Logger.quickLog("CommonResources", "block size %d not used: a multiple of 32 up to 256 is", blockSize);
      }
    }
    return m_DeviceInterface.engine();
  }
  void installPlugIn(const std::string& name) { m_Installed.push_back(name); }
  const std::vector<std::string>& installedPlugIns() const { return m_Installed; }
  uint32_t seed = 1;
  int blockSize = 0;  // from customBlockSize / BlockDim; 0: the engine's default

 private:
  bool m_Initialized = false;
  UtilityConfigFile m_Config;
  UtilityLogger m_Logger{50};
  DeviceInterface m_DeviceInterface;
  brt_params m_Params;
  std::vector<std::string> m_Installed;
};

inline CommonResources m_CommonRes;

#define BRT_READ_PARAM(section, key, target, parser)                                                       \
  do {                                                                                                     \
    const std::string _v = m_CommonRes.getConfig()->getSetting(key, section);                             \
    if (!_v.empty()) target = parser(_v);                                                                  \
  } while (0)

// ---------------------------------------------------------------------------
// DeviceArrayWrapper<T>: host image of one engine feature.  The device image
// is the engine's own array; copyArrayFromDevice / copyArrayToDevice move
// the whole feature in agent-id order.
// Feature::User is a plugin's own per-agent array: registered with the engine
// (brt_engine_add_array), which moves it with the agents at every reorder;
// kernels find it as brt_arrays::user[getUserArrayId()].
enum class Feature { Position, Forward, SmoothAccel, Features, SimilarityStats, Hash, CellStart, NeighList, SteerForce, User };

template <class Type>
class DeviceArrayWrapper {
 public:
  DeviceArrayWrapper(Feature feature, int size, int dimension = 1)
      : m_Feature(feature), m_Size(size), m_Dimension(dimension), m_Host((size_t)size * dimension) {
    // every feature but the cell starts holds one row per agent, and the
    // engine copies all of them to and from the host image
    if (feature != Feature::CellStart && (uint32_t)size != m_CommonRes.params().numBodies)
      throw std::runtime_error("DeviceArrayWrapper: this feature holds one element per agent (size = numBodies)");
    if (feature == Feature::User)
      check(brt_engine_add_array(m_CommonRes.engine(), (uint32_t)(sizeof(Type) * dimension), &m_ArrayId),
            "brt_engine_add_array");
  }
  // The reference's constructor for a plugin's own array
  // (DeviceArrayWrapper.h:74-77): a per-agent array registered with the
  // engine (Feature::User).  Double buffering is internal to the engine and
  // there is no VBO (headless buffers), so the last two flags are accepted
  // and ignored; size must be the engine's agent count.
  DeviceArrayWrapper(DeviceInterface* /*deviceInterface*/, int size, int dimension = 1,
                     bool /*useDoubleBufferingOnDevice*/ = true, bool /*useVbo*/ = false)
      : DeviceArrayWrapper(Feature::User, size, dimension) {}
  uint32_t getUserArrayId() const { return m_ArrayId; }
  Type* getHostArray() { return m_Host.data(); }
  int getSize() const { return m_Size; }
  int getElementBytesCount() const { return (int)sizeof(Type) * m_Dimension; }
  int getBytesCount() const { return getElementBytesCount() * m_Size; }
  Type getHostArrayElement(int index, bool copyFromDevice = false) {
    if (copyFromDevice) copyArrayFromDevice();
    return m_Host[(size_t)index * m_Dimension];
  }
  void setHostArrayElement(int index, const Type* element, bool copyToDevice = false) {
    for (int d = 0; d < m_Dimension; ++d) m_Host[(size_t)index * m_Dimension + d] = element[d];
    if (copyToDevice) copyArrayToDevice();
  }
  void reset(char val) { std::fill((char*)m_Host.data(), (char*)m_Host.data() + m_Host.size() * sizeof(Type), val); }
  void copyArrayFromDevice() {
    brt_engine* e = m_CommonRes.engine();
    void* h = m_Host.data();
    switch (m_Feature) {
      case Feature::Position: check(brt_get_state(e, (float*)h, nullptr, nullptr, nullptr, BRT_MEM_HOST), "getPos"); break;
      case Feature::Forward: check(brt_get_state(e, nullptr, (float*)h, nullptr, nullptr, BRT_MEM_HOST), "getForward"); break;
      case Feature::SmoothAccel: check(brt_get_state(e, nullptr, nullptr, (float*)h, nullptr, BRT_MEM_HOST), "getSmoothAccel"); break;
      case Feature::Features: check(brt_get_state(e, nullptr, nullptr, nullptr, (float*)h, BRT_MEM_HOST), "getFeatures"); break;
      case Feature::SimilarityStats: check(brt_get_similarity_stats(e, (float*)h, BRT_MEM_HOST), "getSimilarityStats"); break;
      case Feature::Hash: {
        std::vector<uint32_t> k(m_Size), id(m_Size);
        check(brt_get_hash(e, k.data(), id.data(), BRT_MEM_HOST), "getHash");
        uint2v* o = (uint2v*)h;
        for (int i = 0; i < m_Size; ++i) o[i] = uint2v{k[i], id[i]};
        break;
      }
      case Feature::CellStart: check(brt_get_cell_ranges(e, (uint32_t*)h, nullptr, BRT_MEM_HOST), "getCellStart"); break;
      case Feature::NeighList: check(brt_get_neighbor_lists(e, (uint32_t*)h, BRT_MEM_HOST), "neighList"); break;
      case Feature::SteerForce: check(brt_get_steer_force(e, (float*)h, BRT_MEM_HOST), "steerForce"); break;
      case Feature::User: check(brt_engine_array_get(e, m_ArrayId, h, BRT_MEM_HOST), "getUserArray"); break;
    }
  }
  void copyArrayToDevice() {
    brt_engine* e = m_CommonRes.engine();
    const float* h = (const float*)m_Host.data();
    switch (m_Feature) {
      case Feature::Position: check(brt_set_state(e, h, nullptr, nullptr, nullptr, BRT_MEM_HOST), "setPos"); break;
      case Feature::Forward: check(brt_set_state(e, nullptr, h, nullptr, nullptr, BRT_MEM_HOST), "setForward"); break;
      case Feature::SmoothAccel: check(brt_set_state(e, nullptr, nullptr, h, nullptr, BRT_MEM_HOST), "setSmoothAccel"); break;
      case Feature::Features: check(brt_set_state(e, nullptr, nullptr, nullptr, h, BRT_MEM_HOST), "setFeatures"); break;
      case Feature::SimilarityStats: check(brt_set_similarity_stats(e, h, BRT_MEM_HOST), "setSimilarityStats"); break;
      case Feature::User: check(brt_engine_array_set(e, m_ArrayId, h, BRT_MEM_HOST), "setUserArray"); break;
      default: throw std::runtime_error("feature is computed by the engine and cannot be written");
    }
  }
  // Double buffering is internal to the engine; kept for source compatibility.
  void swapPosReadWrite() {}
  // The device arrays (DeviceArrayWrapper.h:87-90), for a plugin's own
  // kernels.  A step reads the sorted copy of the state and writes the
  // canonical one, so "read" is the sorted array of the current step (valid
  // after reorderSimData) and "write" the canonical array in the engine's slot
  // order; the engine's own buffers (borrowed, not owned by the wrapper).
  // Features the engine computes (hash, cell starts, lists, steering force)
  // have no separate write array: both calls give the same pointer.
  Type* getReadDeviceArray() { return deviceArray(true); }
  Type* getWriteDeviceArray() { return deviceArray(false); }
  // DeviceArrayWrapper.h:165 stores the repository index a kernel's FETCH
  // uses; kernels here take pointers, so the field receives the user array
  // id (Feature::User) or the feature's number, for source compatibility.
  void bindToField(int& field) { field = m_Feature == Feature::User ? (int)m_ArrayId : (int)m_Feature; }

 private:
  Type* deviceArray(bool read) {
    brt_arrays a;
    check(brt_engine_get_arrays(m_CommonRes.engine(), &a), "brt_engine_get_arrays");
    void* p = nullptr;
    switch (m_Feature) {
      case Feature::Position: p = read ? a.sorted_pos4 : a.pos4; break;
      case Feature::Forward: p = read ? a.sorted_forward4 : a.forward4; break;
      case Feature::SmoothAccel: p = read ? a.sorted_smooth_accel4 : a.smooth_accel4; break;
      case Feature::Features: p = read ? a.sorted_features : a.features; break;
      case Feature::CellStart: p = (void*)a.cell_start; break;
      case Feature::NeighList: p = (void*)a.neighbor_lists; break;
      case Feature::SteerForce: p = a.steer4; break;
      case Feature::User: p = m_ArrayId < a.num_user ? a.user[m_ArrayId] : nullptr; break;
      default: break;
    }
    if (!p) throw std::runtime_error("this feature has no device array in the engine's view");
    return static_cast<Type*>(p);
  }

  Feature m_Feature;
  int m_Size, m_Dimension;
  std::vector<Type> m_Host;
  uint32_t m_ArrayId = 0;
};

// ---------------------------------------------------------------------------
// SimEnginePlugIn / DummyPlugIn (Core/include/SimEnginePlugIn.h:79-200).
class SimEnginePlugIn {
 public:
  virtual ~SimEnginePlugIn() {}
  virtual const std::string name() = 0;
  virtual const DependenciesList plugInDependencies() = 0;
  virtual void reset() = 0;
  virtual void update(const float elapsedTime) = 0;

 protected:
  // Dependency check of Core/src/SimEnginePlugIn.cpp:69-116, throwing
  // instead of exiting.
  void installPlugIn() {
    for (const std::string& dep : plugInDependencies()) {
      bool found = false;
      for (const std::string& p : m_CommonRes.installedPlugIns()) found = found || p == dep;
      if (!found) throw std::runtime_error("missing plugIn dependency " + dep + " of " + name());
    }
    m_CommonRes.installPlugIn(name());
  }
};

class DummyPlugIn : public SimEnginePlugIn {
 public:
  const std::string name() override { return "PlugInRoot"; }
  const DependenciesList plugInDependencies() override { return {}; }
  void reset() override {}
  void update(const float) override {}
};

// ---------------------------------------------------------------------------
// Body3DPlugIn (PlugIns/Body/include/Body3DPlugIn.h:105-129)
template <class Super>
class Body3DPlugIn : public Super {
 public:
  Body3DPlugIn() {
    brt_params& p = m_CommonRes.params();
    const std::string s = "Body3DPlugIn";
    BRT_READ_PARAM(s, "numBodies", p.numBodies, parseInt);
    if (parseBool(m_CommonRes.getConfig()->getSetting("isBodyNumExponent", s))) p.numBodies = 1u << p.numBodies;
    BRT_READ_PARAM(s, "commonRadius", p.commonRadius, parseFloat);
    BRT_READ_PARAM(s, "use2DProjection", p.use2DProjection, parseBool);
    SimEnginePlugIn::installPlugIn();
  }
  const std::string name() override { return "Body3DPlugIn"; }
  const DependenciesList plugInDependencies() override { return {}; }
  void reset() override { Super::reset(); }
  void update(const float t) override { Super::update(t); }
};

// EnvGrid3DPlugIn (PlugIns/EnvGrid3D/include/EnvGrid3DPlugIn.h:56-140)
template <class Super>
class EnvGrid3DPlugIn : public Super {
 public:
  EnvGrid3DPlugIn() {
    brt_params& p = m_CommonRes.params();
    const std::string s = "EnvGrid3DPlugIn";
    float cell[3] = {p.cellSize, p.cellSize, p.cellSize};
    const std::string cs = m_CommonRes.getConfig()->getSetting("cellSize", s);
    if (!cs.empty()) { parseFloat3(cs, cell); p.cellSize = cell[0]; }
    BRT_READ_PARAM(s, "worldSize", p.worldSize, parseFloat);
    // setupWorldRadius (EnvGrid3DPlugIn.h:421-470).  The reference's box spans
    // center -/+ worldRadius; with keepDensity its radius is
    // (numBodies / density)^(1/3) / 2 (the square root in 2D, bodiesDensity2D).
    // Here the periodic cube's side is twice that radius, rounded up to whole
    // cells (the periodic grid needs an integer number of cells, at least 3).
    // An explicit worldSize wins.  worldCenter and lockWorldProportions have
    // no meaning for the periodic cube and are not read.
    UtilityConfigFile* c = m_CommonRes.getConfig();
    if (!c->has("worldSize", s)) {
      float side = 0.0f;
      if (parseBool(c->getSetting("keepDensity", s))) {
        const char* key = p.use2DProjection ? "bodiesDensity2D" : "bodiesDensity3D";
        const float d = c->has(key, s) ? parseFloat(c->getSetting(key, s)) : 0.0f;
        if (d > 0.0f) side = std::pow((float)p.numBodies / d, p.use2DProjection ? 0.5f : 0.33333f);
      } else if (c->has("worldRadius", s)) {
        float r[3] = {0.0f, 0.0f, 0.0f};
        parseFloat3(c->getSetting("worldRadius", s), r);
        side = 2.0f * std::max(r[0], std::max(r[1], r[2]));
      }
      if (side > 0.0f) p.worldSize = std::max(3.0f, std::ceil(side / p.cellSize)) * p.cellSize;
    }
    // setupMaxBodiesPerCell (EnvGrid3DPlugIn.h:537-562): the configured cap,
    // or with useAutomaticMaxBodiesPerCell the upper bound
    // 1 + cellVolume / bodyVolume, bodyVolume = 4.1866 r^3 of the body radius
    if (parseBool(m_CommonRes.getConfig()->getSetting("useAutomaticMaxBodiesPerCell", s))) {
      const float cellVolume = cell[0] * cell[1] * cell[2];
      const float bodyVolume = 4.1866f * p.commonRadius * p.commonRadius * p.commonRadius;
      if (bodyVolume > 0.0f) p.maxBodiesPerCell = (uint32_t)(int)(1.0f + cellVolume / bodyVolume);
    } else {
      BRT_READ_PARAM(s, "maxBodiesPerCell", p.maxBodiesPerCell, parseInt);
    }
    SimEnginePlugIn::installPlugIn();
  }
  const std::string name() override { return "EnvGrid3DPlugIn"; }
  const DependenciesList plugInDependencies() override { return {"Body3DPlugIn"}; }
  // EnvGrid3DPlugIn::reset (:225-275): positions uniform in the world.
  void reset() override {
    Super::reset();
    brt_params& p = m_CommonRes.params();
    std::mt19937 rng(m_CommonRes.seed);
    std::uniform_real_distribution<float> u(0.0f, p.worldSize);
    DeviceArrayWrapper<float4v>* pos = getPos();
    for (uint32_t i = 0; i < p.numBodies; ++i) {
      float4v v{u(rng), u(rng), u(rng), 1.0f};
      for (float* c : {&v.x, &v.y, &v.z}) if (*c >= p.worldSize) *c = 0.0f;
      pos->setHostArrayElement((int)i, &v);
    }
    pos->copyArrayToDevice();
  }
  void update(const float t) override { Super::update(t); }
  void reorderSimData() { check(brt_reorder_sim_data(m_CommonRes.engine()), "reorderSimData"); }
  DeviceArrayWrapper<float4v>* getPos() {
    if (!m_Pos) m_Pos.reset(new DeviceArrayWrapper<float4v>(Feature::Position, (int)m_CommonRes.params().numBodies));
    return m_Pos.get();
  }
  DeviceArrayWrapper<uint2v>* getHash() {
    if (!m_Hash) m_Hash.reset(new DeviceArrayWrapper<uint2v>(Feature::Hash, (int)m_CommonRes.params().numBodies));
    return m_Hash.get();
  }
  // Agent id of the agent at sorted slot `index`.
  uint getSortedIndex(uint index, bool copyFromDevice = true) { return getHash()->getHostArrayElement((int)index, copyFromDevice).y; }
  // addToFeaturesToReorder (EnvGrid3DPlugIn.h:101): every engine feature
  // and every plugin array (Feature::User, registered when it is built) is
  // already reordered with the agents at each step, so this only checks the
  // wrapper is one of those.
  template <class T>
  void addToFeaturesToReorder(DeviceArrayWrapper<T>* feature, const void* /*type*/ = nullptr) {
    if (!feature) throw std::runtime_error("addToFeaturesToReorder: no feature");
  }

 protected:
  std::unique_ptr<DeviceArrayWrapper<float4v>> m_Pos;
  std::unique_ptr<DeviceArrayWrapper<uint2v>> m_Hash;
};

// Proximity3DPlugIn (PlugIns/Proximity3D/include/Proximity3DPlugIn.h:56-110)
template <class Super>
class Proximity3DPlugIn : public Super {
 public:
  Proximity3DPlugIn() {
    brt_params& p = m_CommonRes.params();
    const std::string s = "Proximity3DPlugIn";
    BRT_READ_PARAM(s, "useKnn", p.useKnn, parseBool);
    BRT_READ_PARAM(s, "maxNeighbors", p.maxNeighbors, parseInt);
    BRT_READ_PARAM(s, "commonSearchRadius", p.commonSearchRadius, parseFloat);
    if (parseBool(m_CommonRes.getConfig()->getSetting("useCellSizeAsSearchRadius", s))) p.commonSearchRadius = p.cellSize;
    // searchDepth (Proximity3DPlugIn.h:120-125): the cells scanned on each
    // side of the home cell.  The engine scans the 27 cells of depth 1 1 1
    // (cellSize >= radius); other depths are refused.
    UtilityConfigFile* c = m_CommonRes.getConfig();
    if (c->has("searchDepth", s)) {
      std::istringstream in(c->getSetting("searchDepth", s));
      int d[3] = {1, 1, 1};
      in >> d[0] >> d[1] >> d[2];
      if (d[0] != 1 || d[1] != 1 || d[2] != 1)
        throw std::runtime_error("Proximity3DPlugIn: searchDepth must be 1 1 1 (the 27-cell neighbourhood)");
    }
    // customBlockSize (Proximity3DPlugIn.h:131-134), or DeviceInterface's
    // BlockDim: the flock kernel's threads per block.  useSplittedNeigCalc and
    // useForwardVBO choose reference code paths (a split list kernel, GL
    // buffers) that have no counterpart; they are not read.
    if (c->has("customBlockSize", s)) m_CommonRes.blockSize = parseInt(c->getSetting("customBlockSize", s));
    else if (c->has("BlockDim", "DeviceInterface")) m_CommonRes.blockSize = parseInt(c->getSetting("BlockDim", "DeviceInterface"));
    SimEnginePlugIn::installPlugIn();
  }
  const std::string name() override { return "Proximity3DPlugIn"; }
  const DependenciesList plugInDependencies() override { return {"Body3DPlugIn", "EnvGrid3DPlugIn"}; }
  void reset() override { Super::reset(); }
  void update(const float t) override { Super::update(t); }
  void computeNeighborhoods() { check(brt_compute_neighborhoods(m_CommonRes.engine()), "computeNeighborhoods"); }
  DeviceArrayWrapper<uint>* getCellStart() {
    if (!m_CellStart) {
      uint32_t cells = 0;
      check(brt_engine_num_cells(m_CommonRes.engine(), &cells), "num_cells");
      m_CellStart.reset(new DeviceArrayWrapper<uint>(Feature::CellStart, (int)cells));
    }
    return m_CellStart.get();
  }
  DeviceArrayWrapper<uint>* getNeighList() {
    if (!m_NeighList) {
      uint32_t stride = 0;
      check(brt_neighbor_list_stride(m_CommonRes.engine(), &stride), "list_stride");
      m_NeighList.reset(new DeviceArrayWrapper<uint>(Feature::NeighList, (int)m_CommonRes.params().numBodies, (int)stride));
    }
    return m_NeighList.get();
  }

 protected:
  std::unique_ptr<DeviceArrayWrapper<uint>> m_CellStart;
  std::unique_ptr<DeviceArrayWrapper<uint>> m_NeighList;
};

// OpenSteerWrapperPlugIn (PlugIns/OpenSteerWrapper/include/OpenSteerWrapperPlugIn.h:54-120)
template <class Super>
class OpenSteerWrapperPlugIn : public Super {
 public:
  OpenSteerWrapperPlugIn() {
    brt_params& p = m_CommonRes.params();
    const std::string s = "OpenSteerWrapperPlugIn";
    UtilityConfigFile* c = m_CommonRes.getConfig();
    if (c->has("separationParams", s)) parseFloat3(c->getSetting("separationParams", s), p.separationParams);
    if (c->has("cohesionParams", s)) parseFloat3(c->getSetting("cohesionParams", s), p.cohesionParams);
    if (c->has("alignmentParams", s)) parseFloat3(c->getSetting("alignmentParams", s), p.alignmentParams);
    BRT_READ_PARAM(s, "commonMass", p.commonMass, parseFloat);
    BRT_READ_PARAM(s, "commonMaxSpeed", p.commonMaxSpeed, parseFloat);
    BRT_READ_PARAM(s, "commonMaxForce", p.commonMaxForce, parseFloat);
    BRT_READ_PARAM(s, "commonSensingMinRadius", p.commonSensingMinRadius, parseFloat);
    // avoidBaseParams with the defaults of OpenSteerWrapperPlugIn.h:141-150
    if (c->has("avoidBaseParams", s)) parseFloat3(c->getSetting("avoidBaseParams", s), avoidBaseParams);
    if (avoidBaseParams[0] == 0.0f) {
      avoidBaseParams[0] = 500.0f;
      avoidBaseParams[1] = 500.0f;
      avoidBaseParams[2] = 1000.0f;
    }
    SimEnginePlugIn::installPlugIn();
  }
  // hOpenSteerWrapperParams.avoidBase / avoidBaseParams: set by the
  // application before steerForMoveAwayBaseTarget, as the reference's do.
  float avoidBase[3] = {0.0f, 0.0f, 0.0f};
  float avoidBaseParams[3] = {0.0f, 0.0f, 0.0f};
  const std::string name() override { return "OpenSteerWrapperPlugIn"; }
  const DependenciesList plugInDependencies() override { return {"EnvGrid3DPlugIn", "Proximity3DPlugIn"}; }
  // OpenSteerWrapperPlugIn::reset (:195-263): random unit forward, w = maxSpeed.
  void reset() override {
    Super::reset();
    brt_params& p = m_CommonRes.params();
    std::mt19937 rng(m_CommonRes.seed + 1);
    std::normal_distribution<float> g(0.0f, 1.0f);
    DeviceArrayWrapper<float4v>* fwd = getForward();
    DeviceArrayWrapper<float4v>* acc = getSmoothAccel();
    for (uint32_t i = 0; i < p.numBodies; ++i) {
      float x = g(rng), y = g(rng), z = g(rng);
      const float l = std::sqrt(x * x + y * y + z * z);
      float4v f{x / l, y / l, z / l, p.commonMaxSpeed}, a{0, 0, 0, 0};
      fwd->setHostArrayElement((int)i, &f);
      acc->setHostArrayElement((int)i, &a);
    }
    fwd->copyArrayToDevice();
    acc->copyArrayToDevice();
  }
  void update(const float t) override { Super::update(t); }
  void resetSteerForce() { check(brt_reset_steer_force(m_CommonRes.engine()), "resetSteerForce"); }
  void computeSeparations() { check(brt_compute_separations(m_CommonRes.engine()), "computeSeparations"); }
  void computeAlignments() { check(brt_compute_alignments(m_CommonRes.engine()), "computeAlignments"); }
  void computeCohesions() { check(brt_compute_cohesions(m_CommonRes.engine()), "computeCohesions"); }
  void computeSeekingsWorldCenter() { check(brt_compute_seekings_world_center(m_CommonRes.engine()), "computeSeekingsWorldCenter"); }
  void steerAndSlowToAvoidNeighbors() {
    check(brt_steer_and_slow_to_avoid_neighbors(m_CommonRes.engine()), "steerAndSlowToAvoidNeighbors");
  }
  void steerForMoveAwayBaseTarget() {
    check(brt_steer_for_move_away_base_target(m_CommonRes.engine(), avoidBase, avoidBaseParams),
          "steerForMoveAwayBaseTarget");
  }
  void applySteeringForces(float elapsedTime) { check(brt_apply_steering_forces(m_CommonRes.engine(), elapsedTime), "applySteeringForces"); }
  DeviceArrayWrapper<float4v>* getForward() {
    if (!m_Forward) m_Forward.reset(new DeviceArrayWrapper<float4v>(Feature::Forward, (int)m_CommonRes.params().numBodies));
    return m_Forward.get();
  }
  DeviceArrayWrapper<float4v>* getSmoothAccel() {
    if (!m_Accel) m_Accel.reset(new DeviceArrayWrapper<float4v>(Feature::SmoothAccel, (int)m_CommonRes.params().numBodies));
    return m_Accel.get();
  }
  DeviceArrayWrapper<float4v>* getSteerForce() {
    if (!m_Steer) m_Steer.reset(new DeviceArrayWrapper<float4v>(Feature::SteerForce, (int)m_CommonRes.params().numBodies));
    return m_Steer.get();
  }
  // The whole per-frame update of BehaveRT_Flocking.cpp:177-199 as one call
  // (fused kernel; nsteps > 1 runs a captured CUDA graph).
  void step(float elapsedTime, uint32_t nsteps = 1) { check(brt_step(m_CommonRes.engine(), elapsedTime, nsteps), "brt_step"); }
  // calcInverseHash (OpenSteerWrapperPlugIn.h:278-284, calcInverseHashD,
  // envgrid3d_kernel.cu:70-78), the reference's host-debugging map from agent
  // id to the agent's sorted slot, built on the host from the sorted hash.
  void calcInverseHash() {
    const uint32_t n = m_CommonRes.params().numBodies;
    std::vector<uint32_t> keys(n), ids(n);
    check(brt_get_hash(m_CommonRes.engine(), keys.data(), ids.data(), BRT_MEM_HOST), "calcInverseHash");
    m_InverseHash.assign(n, 0u);
    for (uint32_t i = 0; i < n; ++i)
      if (ids[i] < n) m_InverseHash[ids[i]] = i;
  }
  const std::vector<uint32_t>& getInverseHash() const { return m_InverseHash; }

 protected:
  std::unique_ptr<DeviceArrayWrapper<float4v>> m_Forward, m_Accel, m_Steer;
  std::vector<uint32_t> m_InverseHash;
};

// BehaviorClusteringPlugIn (PlugIns/BehaviorClustering/include/BehaviorClusteringPlugIn.h:60-230)
template <class Super>
class BehaviorClusteringPlugIn : public Super {
 public:
  BehaviorClusteringPlugIn() {
    brt_params& p = m_CommonRes.params();
    const std::string s = "BehaviorClusteringPlugIn";
    UtilityConfigFile* c = m_CommonRes.getConfig();
    BRT_READ_PARAM(s, "featuresCount", p.featuresCount, parseInt);
    if (c->has("clusteringForceParams", s)) parseFloat3(c->getSetting("clusteringForceParams", s), p.clusteringForceParams);
    if (c->has("alignmentClusteringForceParams", s))
      parseFloat3(c->getSetting("alignmentClusteringForceParams", s), p.alignmentClusteringForceParams);
    if (c->has("similarityStatsParams", s)) parseFloat3(c->getSetting("similarityStatsParams", s), p.similarityStatsParams);
    BRT_READ_PARAM(s, "featureRelaxRate", p.featureRelaxRate, parseFloat);
    BRT_READ_PARAM(s, "iterationLP", m_IterationLP, parseInt);
    BRT_READ_PARAM(s, "sameClusterMaxRadius", m_SameClusterMaxRadius, parseFloat);
    SimEnginePlugIn::installPlugIn();
  }
  const std::string name() override { return "BehaviorClusteringPlugIn"; }
  const DependenciesList plugInDependencies() override {
    return {"Body3DPlugIn", "EnvGrid3DPlugIn", "Proximity3DPlugIn", "OpenSteerWrapperPlugIn"};
  }
  void reset() override {
    Super::reset();
    brt_params& p = m_CommonRes.params();
    if (!p.featuresCount) return;
    std::mt19937 rng(m_CommonRes.seed + 2);
    std::uniform_real_distribution<float> u(0.0f, 1.0f);
    DeviceArrayWrapper<float>* f = getFeaturesVector();
    std::vector<float> v(p.featuresCount);
    for (uint32_t i = 0; i < p.numBodies; ++i) {
      for (float& x : v) x = u(rng);
      f->setHostArrayElement((int)i, v.data());
    }
    f->copyArrayToDevice();
  }
  void update(const float t) override { Super::update(t); }
  void steerForClustering() { check(brt_steer_for_clustering(m_CommonRes.engine()), "steerForClustering"); }
  // computeClusterMembership / analyzeClusterHitRate (BehaviorClusteringPlugIn.h
  // :828-894) with the reference's iterationLP = 10 and sameClusterMaxRadius =
  // 1.5 unless the config section sets them.
  void computeClusterMembership() {
    check(brt_compute_cluster_membership(m_CommonRes.engine(), (uint32_t)m_IterationLP), "computeClusterMembership");
  }
  void analyzeClusterHitRate() {
    check(brt_analyze_cluster_hit_rate(m_CommonRes.engine(), m_SameClusterMaxRadius), "analyzeClusterHitRate");
  }
  // (label, hit rate, mean close-neighbour label, unused) per agent id
  std::vector<float4v> getClusterMembership() {
    std::vector<float4v> out(m_CommonRes.params().numBodies);
    check(brt_get_cluster_membership(m_CommonRes.engine(), (float*)out.data(), BRT_MEM_HOST), "getClusterMembership");
    return out;
  }
  // mergeClusters (BehaviorClusteringPlugIn.h:930-952, kernel
  // BehaviorClustering_MergeClusters_kernel, BehaviorClustering_kernel.cu:
  // 697-742): the agents whose leader is one of the two leaders head for the
  // other leader at the maximum speed, forward = normalize(other leader's
  // position - own leader's position); the rest keep their forward.  Leaders
  // are labels of the last computeClusterMembership (sorted slots of that
  // step), as the reference's mergeClusterLeaders; equal leaders do nothing.
  // Runs on the host over the engine's state (an interactive operation of
  // the demo, not part of a step).
  void mergeClusters(int leaderA, int leaderB) {
    if (leaderA == leaderB) return;
    brt_engine* e = m_CommonRes.engine();
    const uint32_t n = m_CommonRes.params().numBodies;
    const std::vector<float4v> member = getClusterMembership();
    std::vector<uint32_t> keys(n), ids(n);
    check(brt_get_hash(e, keys.data(), ids.data(), BRT_MEM_HOST), "mergeClusters");
    std::vector<float4v> pos(n), fwd(n);
    check(brt_get_state(e, (float*)pos.data(), (float*)fwd.data(), nullptr, nullptr, BRT_MEM_HOST), "mergeClusters");
    auto leaderPos = [&](int leader) -> float4v {
      if (leader < 0 || (uint32_t)leader >= n) throw std::runtime_error("mergeClusters: leader out of range");
      return pos[ids[(uint32_t)leader]];
    };
    const float4v pa = leaderPos(leaderA), pb = leaderPos(leaderB);
    const float speed = m_CommonRes.params().commonMaxSpeed;
    for (uint32_t id = 0; id < n; ++id) {
      const int mine = (int)member[id].x;
      if (mine != leaderA && mine != leaderB) continue;
      const float4v& from = mine == leaderA ? pa : pb;
      const float4v& to = mine == leaderA ? pb : pa;
      const float dx = to.x - from.x, dy = to.y - from.y, dz = to.z - from.z;
      const float inv = 1.0f / std::sqrt(dx * dx + dy * dy + dz * dz);
      fwd[id] = float4v{dx * inv, dy * inv, dz * inv, speed};
    }
    check(brt_set_state(e, nullptr, (const float*)fwd.data(), nullptr, nullptr, BRT_MEM_HOST), "mergeClusters");
  }
  // freezeClusters (BehaviorClusteringPlugIn.h:958-967): the reference's
  // freeze kernel (BehaviorClustering_kernel.cu:749-757) has an empty body,
  // so the operation changes nothing.
  void freezeClusters(int /*leader*/) {}
  DeviceArrayWrapper<float>* getFeaturesVector() {
    if (!m_Features)
      m_Features.reset(new DeviceArrayWrapper<float>(Feature::Features, (int)m_CommonRes.params().numBodies,
                                                      (int)m_CommonRes.params().featuresCount));
    return m_Features.get();
  }

 protected:
  std::unique_ptr<DeviceArrayWrapper<float>> m_Features;
  int m_IterationLP = 10;
  float m_SameClusterMaxRadius = 1.5f;
};

// SchoolingPlugIn (PlugIns/Schooling/include/SchoolingPlugIn.h:60-299): the
// install-time constants of the reference (SchoolingPlugIn.h:119-148), each
// overridable from the [SchoolingPlugIn] config section; mode 1 makes the
// fused step run animateSchool, mode 2 the repulsion / attraction-orientation
// / movement sequence.  The random deviation comes from a seeded
// counter-based generator (key "seed") instead of a time-seeded Mersenne
// Twister.
template <class Super>
class SchoolingPlugIn : public Super {
 public:
  SchoolingPlugIn() {
    brt_params& p = m_CommonRes.params();
    brt_schooling_params& sc = p.schooling;
    sc.mode = 1;
    sc.r_p = p.commonSearchRadius;
    const std::string s = "SchoolingPlugIn";
    BRT_READ_PARAM(s, "mode", sc.mode, parseInt);
    BRT_READ_PARAM(s, "theta", sc.theta, parseFloat);
    BRT_READ_PARAM(s, "delta", sc.delta, parseFloat);
    BRT_READ_PARAM(s, "r_r", sc.r_r, parseFloat);
    BRT_READ_PARAM(s, "r_p", sc.r_p, parseFloat);
    BRT_READ_PARAM(s, "eta", sc.eta, parseFloat);
    BRT_READ_PARAM(s, "w_a", sc.w_a, parseFloat);
    BRT_READ_PARAM(s, "w_o", sc.w_o, parseFloat);
    BRT_READ_PARAM(s, "s", sc.s, parseFloat);
    BRT_READ_PARAM(s, "randomDeviationWeight", sc.randomDeviationWeight, parseFloat);
    BRT_READ_PARAM(s, "seed", sc.seed, parseInt);
    SimEnginePlugIn::installPlugIn();
  }
  const std::string name() override { return "SchoolingPlugIn"; }
  const DependenciesList plugInDependencies() override {
    return {"Body3DPlugIn", "EnvGrid3DPlugIn", "Proximity3DPlugIn", "OpenSteerWrapperPlugIn"};
  }
  // Forward speeds are the constant speed s.
  void reset() override {
    Super::reset();
    brt_params& p = m_CommonRes.params();
    DeviceArrayWrapper<float4v>* fwd = this->getForward();
    float4v* host = fwd->getHostArray();
    for (uint32_t i = 0; i < p.numBodies; ++i) host[i].w = p.schooling.s;
    fwd->copyArrayToDevice();
    // restart the random stream, so a reset replays the same run
    check(brt_engine_set_option(m_CommonRes.engine(), "random_step", 0), "reset random stream");
  }
  void update(const float t) override { Super::update(t); }
  void animateSchool() { check(brt_school_animate(m_CommonRes.engine()), "animateSchool"); }
  void calcRepulsion() { check(brt_school_repulsion(m_CommonRes.engine()), "calcRepulsion"); }
  void calcAttractionOrientation() {
    check(brt_school_attraction_orientation(m_CommonRes.engine()), "calcAttractionOrientation");
  }
  void calcMovement() { check(brt_school_movement(m_CommonRes.engine()), "calcMovement"); }
};

}  // namespace BehaveRT
