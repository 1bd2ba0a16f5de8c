// Host runtime and C ABI of the LST object-building chain on one GPU.
//
// An event set (lst_event) owns one device arena holding N event slots; each
// slot carries the complete object stores of one event at their static
// capacities, so nothing is allocated while events run.  Stages are launched
// with gridDim.y = number of events, so the per-event calls (one slot) and the
// batched calls (many slots) run the same kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <sstream>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include "es.h"
#include "lst_b200.h"
#include "lst_fields.h"
#include "lst_kernels.cuh"

namespace {

  thread_local std::string g_lastError;

  int setError(const std::string& msg) {
    try {
      g_lastError = msg;
    } catch (...) {
    }
    return -1;
  }

  // Records "<prefix><what>" without letting an allocation failure escape.
  int abiFail(const char* prefix, const char* what) noexcept {
    try {
      g_lastError = std::string(prefix) + what;
    } catch (...) {
    }
    return -1;
  }

  // Live event setups per device; the cached device address of the static
  // output staging (lst_batch_get_output_static) is dropped when the last
  // one on a device is freed.  Defined with that staging below.
  void staticOutputDeviceRetain(int device);
  void staticOutputDeviceRelease(int device);

  // No C++ exception crosses the C ABI: every entry point runs its body
  // between LST_ABI_TRY and LST_ABI_CATCH_INT (or _VOID), which turn a host
  // allocation failure or any other exception into a -1 status and a message.
#define LST_ABI_TRY try {
#define LST_ABI_CATCH_INT                          \
  }                                                \
  catch (const std::bad_alloc&) {                  \
    return abiFail("out of host memory", "");      \
  }                                                \
  catch (const std::exception& e_) {               \
    return abiFail("internal error: ", e_.what()); \
  }                                                \
  catch (...) {                                    \
    return abiFail("internal error", "");          \
  }
#define LST_ABI_CATCH_VOID \
  }                        \
  catch (...) {            \
  }

  int cudaFail(cudaError_t e, const char* what) {
    return setError(std::string(what) + ": " + cudaGetErrorString(e));
  }

#define LST_CUDA(call)                 \
  do {                                 \
    cudaError_t e_ = (call);           \
    if (e_ != cudaSuccess)             \
      return cudaFail(e_, #call);      \
  } while (0)

  // Launches a kernel on stream `s` and returns an error naming it if the
  // launch is rejected.
  // With profiling on, each launch is bracketed by two CUDA events on the
  // same stream (see lst_event_set_profiling).
#define LST_LAUNCH(kernel, grid, block, ...) LST_LAUNCH_SMEM(kernel, grid, block, 0, __VA_ARGS__)
#define LST_LAUNCH_SMEM(kernel, grid, block, smem, ...)        \
  do {                                                         \
    cudaGetLastError(); /* drop a stale non-sticky error */    \
    cudaEvent_t p0_ = nullptr;                                 \
    if (ev->profiling && (p0_ = profEvent(ev)))                \
      cudaEventRecord(p0_, s);                                 \
    kernel<<<(grid), (block), (smem), s>>>(__VA_ARGS__);       \
    cudaError_t e_ = cudaGetLastError();                       \
    if (e_ != cudaSuccess)                                     \
      return cudaFail(e_, #kernel);                            \
    ++ev->launches;                                            \
    cudaEvent_t p1_ = nullptr;                                 \
    if (p0_ && (p1_ = profEvent(ev))) {                        \
      cudaEventRecord(p1_, s);                                 \
      ev->profile.push_back(ProfRecord{#kernel, p0_, p1_});    \
    }                                                          \
  } while (0)

  // Carves 256-byte-aligned sub-arrays out of one allocation.  With a null
  // base it only measures.
  struct Carver {
    char* base = nullptr;
    size_t off = 0;
    template <typename T>
    T* take(size_t n) {
      off = (off + 255) & ~size_t(255);
      T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
      off += n * sizeof(T);
      return p;
    }
  };

  struct Sizes {
    size_t H, M, L, MD, LS, P, T3, T5, P3, P5, TC;
  };

  void carveEvent(Carver& c, lst::EventView& v, const Sizes& s) {
    const size_t H = s.H, M = s.M, L = s.L, MD = s.MD, LS = s.LS, P = s.P, T3 = s.T3, T5 = s.T5, P3 = s.P3,
                 P5 = s.P5, TC = s.TC;
    (void)H;
#define LST_CARVE(prefix, member, field, type, count) v.member.field = c.take<type>(count);
    LST_EVENT_FIELDS(LST_CARVE)
#undef LST_CARVE
#define LST_CARVE_SCRATCH(field, type, count) v.field = c.take<type>(count);
    LST_SCRATCH_FIELDS(LST_CARVE_SCRATCH)
#undef LST_CARVE_SCRATCH
    v.md.slope = c.take<float>(MD);
    v.md.tanSlope = c.take<float>(MD);
    v.md.slope3 = c.take<float>(MD);
    v.md.anchorPos = c.take<lst::MDPos>(MD);
    v.md.rec = c.take<lst::MDRec>(MD);
    v.sc = c.take<lst::EventScalars>(1);
  }

  struct FieldInfo {
    std::string name;
    size_t elemSize;
    char kind;
  };

  template <typename T>
  constexpr char kindOf() {
    return std::is_floating_point<T>::value ? 'f' : (std::is_signed<T>::value ? 'i' : 'u');
  }

  // Field names ("store.field") and element types in table order.
  const std::vector<FieldInfo>& fieldTable() {
    static const std::vector<FieldInfo> table = [] {
      std::vector<FieldInfo> t;
#define LST_NAME(prefix, member, field, type, count) \
  t.push_back(FieldInfo{std::string(prefix) + #field, sizeof(type), kindOf<type>()});
      LST_EVENT_FIELDS(LST_NAME)
#undef LST_NAME
      return t;
    }();
    return table;
  }

  // Device pointer, length and element size of a named field of one view.
  bool findField(const lst::EventView& v, const Sizes& s, const std::string& name, void*& ptr, size_t& n,
                 size_t& esz) {
    const size_t H = s.H, M = s.M, L = s.L, MD = s.MD, LS = s.LS, P = s.P, T3 = s.T3, T5 = s.T5, P3 = s.P3,
                 P5 = s.P5, TC = s.TC;
    (void)H;
#define LST_FIND(prefix, member, field, type, count) \
  if (name == prefix #field) {                       \
    ptr = (void*)v.member.field;                     \
    n = (count);                                     \
    esz = sizeof(type);                              \
    return true;                                     \
  }
    LST_EVENT_FIELDS(LST_FIND)
#undef LST_FIND
    return false;
  }

  unsigned int ceilDiv(size_t a, size_t b) { return static_cast<unsigned int>((a + b - 1) / b); }

}  // namespace

// ------------------------------------------------------------------ ES
struct lst_es {
  int device = 0;
  lst::EsHost host;
  lst::DeviceES view{};
  void* arena = nullptr;
  size_t arenaBytes = 0;
  bool haveDnn = false;
  unsigned int nEligibleMax = 0;  // lower modules that can seed T5s
  std::vector<float> dnn;
};

namespace {

  template <typename T>
  const T* upload(Carver& c, const std::vector<T>& v, std::vector<std::pair<void*, const void*>>& copies,
                  std::vector<size_t>& sizes) {
    T* p = c.take<T>(std::max<size_t>(v.size(), 1));
    if (c.base && !v.empty()) {
      copies.emplace_back(p, v.data());
      sizes.push_back(v.size() * sizeof(T));
    }
    return p;
  }

  // Lays out (or, with a base, fills) the device copy of the event setup.
  void layoutES(Carver& c, lst_es& es, std::vector<std::pair<void*, const void*>>& copies, std::vector<size_t>& sizes) {
    const lst::EsHost& h = es.host;
    lst::DeviceES& d = es.view;
    lst::Modules& m = d.m;
    m.detIds = upload(c, h.detIds, copies, sizes);
    m.moduleMap = upload(c, h.moduleMap, copies, sizes);
    m.mapdetId = upload(c, h.mapdetId, copies, sizes);
    m.mapIdx = upload(c, h.mapIdx, copies, sizes);
    m.nConnectedModules = upload(c, h.nConnectedModules, copies, sizes);
    m.drdzs = upload(c, h.drdzs, copies, sizes);
    m.dxdys = upload(c, h.dxdys, copies, sizes);
    m.partnerModuleIndices = upload(c, h.partnerModuleIndices, copies, sizes);
    m.layers = upload(c, h.layers, copies, sizes);
    m.rings = upload(c, h.rings, copies, sizes);
    m.modules = upload(c, h.modules, copies, sizes);
    m.rods = upload(c, h.rods, copies, sizes);
    m.subdets = upload(c, h.subdets, copies, sizes);
    m.sides = upload(c, h.sides, copies, sizes);
    m.eta = upload(c, h.eta, copies, sizes);
    m.r = upload(c, h.r, copies, sizes);
    m.isInverted = upload(c, h.isInverted, copies, sizes);
    m.isLower = upload(c, h.isLower, copies, sizes);
    m.isAnchor = upload(c, h.isAnchor, copies, sizes);
    m.moduleType = upload(c, h.moduleType, copies, sizes);
    m.moduleLayerType = upload(c, h.moduleLayerType, copies, sizes);
    m.sdlLayers = upload(c, h.sdlLayers, copies, sizes);
    m.connectedPixels = upload(c, h.connectedPixels, copies, sizes);
    m.geoMapDetId = upload(c, h.geoMapDetId, copies, sizes);
    m.geoMapPhi = upload(c, h.geoMapPhi, copies, sizes);
    m.geoMapIndex = upload(c, h.geoMapIndex, copies, sizes);
    m.nEndCapMap = static_cast<unsigned int>(h.geoMapDetId.size());
    m.nModules = h.nModules;
    m.nLowerModules = h.nLowerModules;
    m.ptCut = h.ptCut;
    d.cpIndex = upload(c, h.connectedPixelsIndex, copies, sizes);
    d.cpSizes = upload(c, h.connectedPixelsSizes, copies, sizes);
    d.cpIndexPos = upload(c, h.connectedPixelsIndexPos, copies, sizes);
    d.cpSizesPos = upload(c, h.connectedPixelsSizesPos, copies, sizes);
    d.cpIndexNeg = upload(c, h.connectedPixelsIndexNeg, copies, sizes);
    d.cpSizesNeg = upload(c, h.connectedPixelsSizesNeg, copies, sizes);
    d.mdOffset = upload(c, h.mdOffset, copies, sizes);
    d.mdCap = upload(c, h.mdCap, copies, sizes);
    d.lsOffset = upload(c, h.lsOffset, copies, sizes);
    d.lsCap = upload(c, h.lsCap, copies, sizes);
    d.t3CapIfUsed = upload(c, h.t3CapIfUsed, copies, sizes);
    d.t5CapIfEligible = upload(c, h.t5CapIfEligible, copies, sizes);
    d.detHashKey = upload(c, h.detHashKey, copies, sizes);
    d.detHashVal = upload(c, h.detHashVal, copies, sizes);
    d.detHashBits = h.detHashBits;
    // The positive- and negative-z pixel maps follow the inclusive one in
    // connectedPixels (SDL/Event.cc:1049-1052).
    const size_t last = lst::kSizeSuperbins - 1;
    d.pixelIndexOffsetPos = h.connectedPixelsIndex[last] + h.connectedPixelsSizes[last];
    d.pixelIndexOffsetNeg = h.connectedPixelsIndexPos[last] + h.connectedPixelsSizesPos[last] + d.pixelIndexOffsetPos;
    d.nTotalMDs = h.nTotalMDs;
    d.nTotalSegments = h.nTotalSegments;
    d.maxTriplets = h.maxTriplets;
    d.maxQuintuplets = h.maxQuintuplets;
    d.nModules = h.nModules;
    d.nLowerModules = h.nLowerModules;
    d.pixelModule = h.pixelModuleIndex;
  }

  int loadWeightsFile(const char* path, std::vector<float>& w) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f.is_open())
      return setError(std::string("cannot open T5 DNN weights ") + path);
    std::streamsize n = f.tellg();
    if (n != static_cast<std::streamsize>(lst::kT5DnnParams * sizeof(float)))
      return setError(std::string("T5 DNN weight file has the wrong size: ") + path);
    f.seekg(0);
    w.resize(lst::kT5DnnParams);
    f.read(reinterpret_cast<char*>(w.data()), n);
    return 0;
  }

  int uploadWeights(lst_es* es) {
    if (es->dnn.size() != lst::kT5DnnParams)
      return setError("T5 DNN weights must hold 2337 values");
    lst::T5DnnWeights w;
    static_assert(sizeof(lst::T5DnnWeights) == lst::kT5DnnParams * sizeof(float), "packed weight struct");
    std::memcpy(&w, es->dnn.data(), sizeof(w));
    LST_CUDA(cudaSetDevice(es->device));
    LST_CUDA(cudaMemcpyToSymbol(lst::c_t5dnn, &w, sizeof(w)));
    LST_CUDA(cudaDeviceSynchronize());
    es->haveDnn = true;
    return 0;
  }

}  // namespace

// ---------------------------------------------------------------- events
namespace {
  struct ProfRecord {
    const char* kernel;
    cudaEvent_t start, stop;
  };
}  // namespace

namespace {
  // Kernels whose launch shape the autotuner picks: warps per block and
  // resident blocks per SM across the batch (the grid holds
  // blocks_per_sm x SMs / events blocks per event).  Their results do not
  // depend on the shape: each module / candidate is processed the same way by
  // whichever warp takes it.
  enum TunedKernel { kTuMD, kTuMDDerived, kTuLS, kTuT3, kTuT5Eval, kTuPix5, kTuPix3, kTuMid5, kTuMid3, kTuCount };
  struct TuneSpec {
    const char* name;  // as it appears in the launch profile
    int maxWarps;      // the kernel's launch bounds / per-warp shared memory
    int defWarps;
  };
  const TuneSpec kTuneSpecs[kTuCount] = {{"kCreateMD", 8, 8},   {"kMDDerived", 8, 8},   {"kCreateLS", 4, 4},
                                         {"kCreateT3", 4, 4},   {"kT5Eval", 4, 4},      {"kPixEval<5>", 4, 4},
                                         {"kPixEval<3>", 4, 4}, {"kPixMid<5>", 4, 4},    {"kPixMid<3>", 4, 4}};
  constexpr int kDefaultBlocksPerSM = 16;
  struct LaunchShape {
    int warps = 4;
    int perSM = kDefaultBlocksPerSM;
  };
}  // namespace

struct lst_event {
  lst_es* es = nullptr;
  int device = 0;
  int nSlots = 0;
  unsigned int maxHits = 0;
  cudaStream_t stream = nullptr;
  bool ownStream = false;
  char* arena = nullptr;
  size_t slotBytes = 0;
  size_t totalBytes = 0;
  Sizes sizes{};
  std::vector<lst::EventView> hv;
  lst::EventView* dv = nullptr;
  int t5Method = LST_T5_DNN;
  int nSM = 148;
  LaunchShape shape[kTuCount];
  // batched-input staging: the last upload's packed events (kind 0: the
  // Event-API layout of lst_batch_upload, 1: CMSSW seeds of
  // lst_batch_upload_seeds) for slots [inboxFirst, inboxFirst + inboxCount)
  unsigned char* inbox = nullptr;          // current input source of ingestInbox
  unsigned long long* dOffsets = nullptr;  //   and its per-slot blob offsets
  unsigned char* ownInbox = nullptr;       // the buffer of lst_batch_upload*
  size_t inboxBytes = 0;
  unsigned long long* ownOffsets = nullptr;
  size_t inboxUsed = 0;
  // double-buffered staging of lst_batch_stage on its own copy stream
  struct StageBuf {
    unsigned char* ptr = nullptr;
    size_t bytes = 0;
    unsigned long long* offsets = nullptr;
    cudaEvent_t ready = nullptr;  // the copy into it has finished
    cudaEvent_t freed = nullptr;  // the last ingest that read it has finished
  } stage[2];
  int stageNext = 0;
  cudaStream_t copyStream = nullptr;
  struct {
    bool pending = false;
    int first = 0, count = 0, kind = 0, buf = 0;
    size_t total = 0;
  } staged;
  bool inboxValid = false;
  int inboxKind = 0;
  int inboxFirst = 0, inboxCount = 0;
  std::vector<unsigned char> hostPack;  // staging of lst_event_prepare_input
  // per-slot counts, contiguous on the device and in pinned host memory
  lst_counts* dCounts = nullptr;
  lst_counts* hCounts = nullptr;
  // track-candidate output staging (grown on demand)
  unsigned long long* dOutOffsets = nullptr;  // 2 * (nSlots + 1)
  unsigned long long* hOutOffsets = nullptr;  // pinned copy
  unsigned char* dOut = nullptr;
  size_t dOutBytes = 0;
  unsigned int* dProbeCount = nullptr;
  // launch accounting and optional per-launch timing
  unsigned long long launches = 0;
  bool profiling = false;
  std::vector<cudaEvent_t> eventPool;
  size_t poolUsed = 0;
  std::vector<ProfRecord> profile;
  // CUDA graphs of lst_batch_run_graph, keyed by (first, count, stages, method)
  struct GraphEntry {
    cudaGraphExec_t exec = nullptr;
    unsigned long long kernels = 0;
  };
  std::map<std::tuple<int, int, int, int, int, unsigned int>, GraphEntry> graphs;
};

namespace {
  // Next timing event of the set's pool (grown on demand); null if the
  // runtime cannot create one, in which case that launch is not timed.
  cudaEvent_t profEvent(lst_event* ev) {
    if (ev->poolUsed == ev->eventPool.size()) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
      }
      ev->eventPool.push_back(e);
    }
    return ev->eventPool[ev->poolUsed++];
  }
}  // namespace

namespace {

  constexpr unsigned int kThreads = 256;
  constexpr unsigned int kResidentBlocks = 148 * 8;

  // Blocks per event for a grid-stride kernel over n items.
  unsigned int blocksFor(size_t n, int count, unsigned int threads = kThreads) {
    unsigned int want = std::max(1u, ceilDiv(n, threads));
    unsigned int cap = std::max(1u, ceilDiv(2 * kResidentBlocks, static_cast<size_t>(std::max(count, 1))));
    return std::min(want, cap);
  }

  int checkSlots(lst_event* ev, int first, int count) {
    if (!ev)
      return setError("null event set");
    if (first < 0 || count < 0 || first + count > ev->nSlots)
      return setError("slot range outside the event set");
    return 0;
  }


  int runReset(lst_event* ev, int first, int count) {
    const lst_es* es = ev->es;
    dim3 g(blocksFor(2 * size_t(es->view.nModules), count), count);
    cudaStream_t s = ev->stream;
    LST_LAUNCH(lst::kResetEvent, g, kThreads, es->view, ev->dv + first);
    return 0;
  }

  int runHitKernels(lst_event* ev, int first, int count) {
    const lst::DeviceES& d = ev->es->view;
    cudaStream_t s = ev->stream;
    LST_LAUNCH(lst::kHitPrep, dim3(blocksFor(ev->maxHits, count), count), kThreads, d, ev->dv + first);
    LST_LAUNCH(lst::kModuleRanges, dim3(blocksFor(d.nLowerModules, count), count), kThreads, d, ev->dv + first);
    return 0;
  }

  int runPixelIngest(lst_event* ev, int first, int count) {
    const lst::DeviceES& d = ev->es->view;
    cudaStream_t s = ev->stream;
    LST_LAUNCH(lst::kPLSHitReset, dim3(blocksFor(lst::kPLSHitBuckets, count), count), kThreads, ev->dv + first);
    LST_LAUNCH(lst::kPixelIngest, dim3(blocksFor(lst::kMaxPixelSegments, count), count), kThreads, d, ev->dv + first);
    return 0;
  }

  // Warp-per-object kernels: blocks of `warps` warps.
  dim3 warpGrid(size_t nObjects, int warps, int count) {
    return dim3(blocksFor(nObjects * 32, count, 32u * warps), count);
  }

  // Tuned warp-per-object kernel k over nObjects per event.
  dim3 tunedWarpGrid(const lst_event* ev, int k, size_t nObjects, int count) {
    const LaunchShape& sh = ev->shape[k];
    const size_t want = std::max<size_t>(1, ceilDiv(nObjects, static_cast<size_t>(sh.warps)));
    const size_t cap = std::max<size_t>(1, ceilDiv(static_cast<size_t>(sh.perSM) * ev->nSM,
                                                   static_cast<size_t>(std::max(count, 1))));
    return dim3(static_cast<unsigned int>(std::min(want, cap)), count);
  }
  // Tuned kernel k striding over a candidate list whose length only the device knows.
  dim3 tunedFlatGrid(const lst_event* ev, int k, int count) {
    const LaunchShape& sh = ev->shape[k];
    const size_t blocks = std::max<size_t>(1, ceilDiv(static_cast<size_t>(sh.perSM) * ev->nSM,
                                                      static_cast<size_t>(std::max(count, 1))));
    return dim3(static_cast<unsigned int>(blocks), count);
  }
  unsigned int tunedThreads(const lst_event* ev, int k) { return 32u * static_cast<unsigned int>(ev->shape[k].warps); }

  int runStage(lst_event* ev, int first, int count, int stage) {
    const lst::DeviceES& d = ev->es->view;
    const lst::EventView* v = ev->dv + first;
    cudaStream_t s = ev->stream;
    const size_t nLower = d.nLowerModules;
    const size_t P = lst::kMaxPixelSegments;
    const dim3 one(1, count);
    switch (stage) {
      case LST_STAGE_MINI_DOUBLETS: {
        // modules per warp task: 8 from 4 events per launch, 4 for fewer, so
        // that a single event still makes enough tasks to fill the GPU
#ifndef LST_MD_MPT
#define LST_MD_MPT 8u
#endif
        const unsigned int mpt = count >= 4 ? LST_MD_MPT : 4u;
        LST_LAUNCH(lst::kTaskCountersReset, dim3(1, count), 32, v);
        LST_LAUNCH(lst::kCreateMD, tunedWarpGrid(ev, kTuMD, ceilDiv(nLower, mpt), count), tunedThreads(ev, kTuMD), d, v,
                   mpt);
        LST_LAUNCH(lst::kMDRanges, dim3(blocksFor(nLower, count), count), kThreads, d, v);
        LST_LAUNCH(lst::kMDDerived, tunedWarpGrid(ev, kTuMDDerived, nLower + 1, count), tunedThreads(ev, kTuMDDerived),
                   d, v);
        break;
      }
      case LST_STAGE_SEGMENTS:
        LST_LAUNCH(lst::kTaskCountersReset, dim3(1, count), 32, v);
        LST_LAUNCH(lst::kCreateLS, tunedWarpGrid(ev, kTuLS, nLower, count), tunedThreads(ev, kTuLS), d, v);
        LST_LAUNCH(lst::kLSRanges, dim3(blocksFor(nLower, count), count), kThreads, d, v);
        LST_LAUNCH(lst::kLSByMD, warpGrid(ceilDiv(nLower, 32), lst::kIdxWarps, count), 32 * lst::kIdxWarps, d, v);
        break;
      case LST_STAGE_TRIPLETS:
        LST_LAUNCH(lst::kT3Offsets, one, 1024, d, v);
        LST_LAUNCH(lst::kTaskCountersReset, dim3(1, count), 32, v);
        LST_LAUNCH(lst::kCreateT3, tunedWarpGrid(ev, kTuT3, nLower, count), tunedThreads(ev, kTuT3), d, v);
        LST_LAUNCH(lst::kT3Ranges, dim3(blocksFor(nLower, count), count), kThreads, d, v);
        LST_LAUNCH(lst::kT3ByMD, warpGrid(ceilDiv(nLower, 32), lst::kIdxWarps, count), 32 * lst::kIdxWarps, d, v);
        break;
      case LST_STAGE_QUINTUPLETS: {
        if (ev->t5Method == LST_T5_DNN && !ev->es->haveDnn)
          return setError("the DNN T5 method needs weights (lst_es_load or lst_es_set_t5dnn_weights)");
        bool useDnn = ev->t5Method == LST_T5_DNN;
        LST_LAUNCH(lst::kT5Eligible, one, 1024, d, v);
        LST_LAUNCH(lst::kT5Prefix, warpGrid(ev->es->nEligibleMax, 8, count), 256, d, v);
        LST_LAUNCH(lst::kT5ModScan, one, 1024, d, v);
        LST_LAUNCH(lst::kT5Pre, dim3(blocksFor(size_t(1) << 20, count), count), kThreads, d, v);
        LST_LAUNCH(lst::kT5Eval, tunedFlatGrid(ev, kTuT5Eval, count), tunedThreads(ev, kTuT5Eval), d, v, useDnn);
        LST_LAUNCH(lst::kT5Walk, warpGrid(ev->es->nEligibleMax, lst::kT5Warps, count), 32 * lst::kT5Warps, d, v,
                   useDnn);
        LST_LAUNCH_SMEM(lst::kT5RankEmit, dim3(1, count), 1024, lst::kT5RankSmem, d, v);
        LST_LAUNCH(lst::kT5Emit, warpGrid(ev->es->nEligibleMax, 8, count), 256, d, v, useDnn);
        LST_LAUNCH(lst::kT5DedupAfterBuild,
                   dim3(blocksFor(size_t(ev->es->nEligibleMax) * lst::kT5DedupThreads / 32, count, lst::kT5DedupThreads),
                        count),
                   lst::kT5DedupThreads,
                   d, v);
        LST_LAUNCH(lst::kT5Ranges, dim3(blocksFor(nLower, count), count), kThreads, d, v);
        break;
      }
      case LST_STAGE_PLS_CLEANING:
        LST_LAUNCH(lst::kPLSCleanHits, dim3(blocksFor(P, count), count), kThreads, d, v, false);
        break;
      case LST_STAGE_PIXEL_QUINTUPLETS:
        LST_LAUNCH(lst::kPixelConnect, dim3(blocksFor(P, count), count), kThreads, d, v);
        LST_LAUNCH(lst::kPixPrefix<5>, warpGrid(P, 8, count), 256, d, v);
        LST_LAUNCH(lst::kPixScan, one, 1024, d, v);
        LST_LAUNCH(lst::kPixPre<5>, dim3(blocksFor(size_t(1) << 20, count), count), kThreads, d, v);
        LST_LAUNCH(lst::kPixMid<5>, tunedFlatGrid(ev, kTuMid5, count), tunedThreads(ev, kTuMid5), d, v);
        LST_LAUNCH(lst::kPixEval<5>, tunedFlatGrid(ev, kTuPix5, count), tunedThreads(ev, kTuPix5), d, v);
        LST_LAUNCH(lst::kPixRankEmit<5>, one, 1024, d, v);
        LST_LAUNCH(lst::kPT5Count, warpGrid(P, lst::kPixWarps, count), 32 * lst::kPixWarps, d, v);
        LST_LAUNCH(lst::kPLSScan, one, 1024, d, v, 0);
        LST_LAUNCH(lst::kPT5Emit, warpGrid(P, lst::kPixWarps, count), 32 * lst::kPixWarps, d, v);
        LST_LAUNCH_SMEM(lst::kPT5DedupHashed, dim3(lst::kPT5DedupBlocks, count), 1024, lst::kPT5DedupSmem, d, v);
        LST_LAUNCH(lst::kPT5Dedup, dim3(blocksFor(lst::kMaxPixelQuintuplets, count, lst::kDedupTile), count),
                   lst::kDedupTile, d, v);
        LST_LAUNCH(lst::kAddPT5TC, one, 1024, d, v);
        break;
      case LST_STAGE_PIXEL_TRIPLETS:
        LST_LAUNCH(lst::kPixelConnect, dim3(blocksFor(P, count), count), kThreads, d, v);
        LST_LAUNCH(lst::kPixPrefix<3>, warpGrid(P, 8, count), 256, d, v);
        LST_LAUNCH(lst::kPixScan, one, 1024, d, v);
        LST_LAUNCH(lst::kPixPre<3>, dim3(blocksFor(size_t(1) << 20, count), count), kThreads, d, v);
        LST_LAUNCH(lst::kPixMid<3>, tunedFlatGrid(ev, kTuMid3, count), tunedThreads(ev, kTuMid3), d, v);
        LST_LAUNCH(lst::kPixEval<3>, tunedFlatGrid(ev, kTuPix3, count), tunedThreads(ev, kTuPix3), d, v);
        LST_LAUNCH(lst::kPixRankEmit<3>, one, 1024, d, v);
        LST_LAUNCH(lst::kPT3Count, warpGrid(P, lst::kPixWarps, count), 32 * lst::kPixWarps, d, v);
        LST_LAUNCH(lst::kPLSScan, one, 1024, d, v, 1);
        LST_LAUNCH(lst::kPT3Emit, warpGrid(P, lst::kPixWarps, count), 32 * lst::kPixWarps, d, v);
        LST_LAUNCH(lst::kPT3Dedup, warpGrid(lst::kMaxPixelTriplets, 8, count), 256, d, v);
        break;
      case LST_STAGE_TRACK_CANDIDATES: {
        const size_t nE = ev->es->nEligibleMax;
        const dim3 eligGrid(ceilDiv(std::max<size_t>(nE, 1) * 32, 256), count);
        LST_LAUNCH(lst::kCrossCleanPT3, dim3(blocksFor(lst::kMaxPixelTriplets, count), count), kThreads, d, v);
        LST_LAUNCH(lst::kAddPT3TC, one, 1024, d, v);
        LST_LAUNCH(lst::kT5Bin, one, 1024, d, v);
        LST_LAUNCH(lst::kT5DedupBinned, dim3(blocksFor(4096, count), count), kThreads, d, v);
        LST_LAUNCH(lst::kT5DedupBeforeTC, dim3(blocksFor(nE * 32, count), count), 256, d, v);
        LST_LAUNCH(lst::kMergeT5Flag, eligGrid, 256, d, v);
        LST_LAUNCH(lst::kCrossCleanT5, eligGrid, 256, d, v);
        LST_LAUNCH(lst::kT5TCCount, eligGrid, 256, d, v);
        LST_LAUNCH(lst::kT5TCScan, one, 1024, d, v);
        LST_LAUNCH(lst::kT5TCEmit, eligGrid, 256, d, v);
        LST_LAUNCH(lst::kT5TCFinish, one, 32, d, v);
        LST_LAUNCH(lst::kPLSBin, one, 1024, d, v);
        LST_LAUNCH(lst::kPLSCleanHits, dim3(blocksFor(P, count), count), kThreads, d, v, true);
        LST_LAUNCH(lst::kPLSCleanNear, dim3(blocksFor(P, count, lst::kPLSCleanTile), count), lst::kPLSCleanTile, d,
                   v);
        LST_LAUNCH(lst::kMergePLSFlag, dim3(blocksFor(P, count), count), kThreads, d, v);
        LST_LAUNCH(lst::kTCCleanInfo, dim3(blocksFor(lst::kMaxTrackCandidates, count), count), kThreads, d, v);
        LST_LAUNCH_SMEM(lst::kCrossCleanPLS, dim3(lst::kXCleanBlocksPerEvent, count), 1024, lst::kXCleanSmem, d, v);
        LST_LAUNCH(lst::kAddPLSTC, one, 1024, d, v);
        break;
      }
      default:
        return setError("unknown stage " + std::to_string(stage));
    }
    return 0;
  }

  int runCounts(lst_event* ev, int first, int count) {
    cudaStream_t s = ev->stream;
    LST_LAUNCH(lst::kCounts, dim3(1, count), 256, ev->es->view, ev->dv + first);
    return 0;
  }

  // Resets slots [first, first + count) and unpacks their packed inputs from
  // the device inbox: the work of addHitToEvent + addPixelSegmentToEvent,
  // preceded for seed events by the conversion of LST::prepareInput.
  int ingestInbox(lst_event* ev, int first, int count) {
    int rc = runReset(ev, first, count);
    if (rc)
      return rc;
    cudaStream_t s = ev->stream;
    const unsigned long long total = ev->inboxUsed;
    if (ev->inboxKind == 1)
      LST_LAUNCH(lst::kPrepareInput, dim3(1 + blocksFor(ev->maxHits, count, 1024), count), 1024, ev->dv + first,
                 ev->inbox, ev->dOffsets + first, total);
    else
      LST_LAUNCH(lst::kUnpack, dim3(blocksFor(ev->maxHits, count), count), kThreads, ev->dv + first, ev->inbox,
                 ev->dOffsets + first, total);
    rc = runHitKernels(ev, first, count);
    if (rc)
      return rc;
    return runPixelIngest(ev, first, count);
  }

  int readCounts(lst_event* ev, int first, int count, lst_counts* out) {
    int rc = runCounts(ev, first, count);
    if (rc)
      return rc;
    LST_CUDA(cudaMemcpyAsync(ev->hCounts, ev->dCounts + first, sizeof(lst_counts) * count, cudaMemcpyDeviceToHost,
                             ev->stream));
    LST_CUDA(cudaStreamSynchronize(ev->stream));
    std::memcpy(out, ev->hCounts, sizeof(lst_counts) * count);
    return 0;
  }

}  // namespace

// ================================================================== C ABI
namespace {

  struct KernelEntry {
    const char* name;
    const void* fn;
  };

  // Every kernel of the library (for launch-resource queries).
  const std::vector<KernelEntry>& kernelTable() {
    static const std::vector<KernelEntry> t = {
        {"kResetEvent", (const void*)lst::kResetEvent},
        {"kHitPrep", (const void*)lst::kHitPrep},
        {"kModuleRanges", (const void*)lst::kModuleRanges},
        {"kPixelIngest", (const void*)lst::kPixelIngest},
        {"kCreateMD", (const void*)lst::kCreateMD},
        {"kMDRanges", (const void*)lst::kMDRanges},
        {"kMDDerived", (const void*)lst::kMDDerived},
        {"kTaskCountersReset", (const void*)lst::kTaskCountersReset},
        {"kCreateLS", (const void*)lst::kCreateLS},
        {"kLSRanges", (const void*)lst::kLSRanges},
        {"kT3Offsets", (const void*)lst::kT3Offsets},
        {"kCreateT3", (const void*)lst::kCreateT3},
        {"kLSByMD", (const void*)lst::kLSByMD},
        {"kT3ByMD", (const void*)lst::kT3ByMD},
        {"kT3Ranges", (const void*)lst::kT3Ranges},
        {"kT5Eligible", (const void*)lst::kT5Eligible},
        {"kT5Prefix", (const void*)lst::kT5Prefix},
        {"kT5ModScan", (const void*)lst::kT5ModScan},
        {"kT5Eval", (const void*)lst::kT5Eval},
        {"kT5Emit", (const void*)lst::kT5Emit},
        {"kT5RankEmit", (const void*)lst::kT5RankEmit},
        {"kT5Walk", (const void*)lst::kT5Walk},
        {"kT5Probe", (const void*)lst::kT5Probe},
        {"kT5DedupAfterBuild", (const void*)lst::kT5DedupAfterBuild},
        {"kT5Ranges", (const void*)lst::kT5Ranges},
        {"kPLSBin", (const void*)lst::kPLSBin},
        {"kPLSHitReset", (const void*)lst::kPLSHitReset},
        {"kPLSCleanHits", (const void*)lst::kPLSCleanHits},
        {"kPLSCleanNear", (const void*)lst::kPLSCleanNear},
        {"kMergePLSFlag", (const void*)lst::kMergePLSFlag},
        {"kPixelConnect", (const void*)lst::kPixelConnect},
        {"kPixPrefix<5>", (const void*)lst::kPixPrefix<5>},
        {"kPixPrefix<3>", (const void*)lst::kPixPrefix<3>},
        {"kPixScan", (const void*)lst::kPixScan},
        {"kPixEval<5>", (const void*)lst::kPixEval<5>},
        {"kPixPre<5>", (const void*)lst::kPixPre<5>},
        {"kT5Pre", (const void*)lst::kT5Pre},
        {"kPixMid<5>", (const void*)lst::kPixMid<5>},
        {"kPixMid<3>", (const void*)lst::kPixMid<3>},
        {"kPixPre<3>", (const void*)lst::kPixPre<3>},
        {"kPixEval<3>", (const void*)lst::kPixEval<3>},
        {"kPixRankEmit<5>", (const void*)lst::kPixRankEmit<5>},
        {"kPixRankEmit<3>", (const void*)lst::kPixRankEmit<3>},
        {"kPT5Count", (const void*)lst::kPT5Count},
        {"kPT5Emit", (const void*)lst::kPT5Emit},
        {"kPLSScan", (const void*)lst::kPLSScan},
        {"kPT5Dedup", (const void*)lst::kPT5Dedup},
        {"kPT5DedupHashed", (const void*)lst::kPT5DedupHashed},
        {"kAddPT5TC", (const void*)lst::kAddPT5TC},
        {"kPT3Count", (const void*)lst::kPT3Count},
        {"kPT3Emit", (const void*)lst::kPT3Emit},
        {"kPT3Dedup", (const void*)lst::kPT3Dedup},
        {"kCrossCleanPT3", (const void*)lst::kCrossCleanPT3},
        {"kAddPT3TC", (const void*)lst::kAddPT3TC},
        {"kT5DedupBeforeTC", (const void*)lst::kT5DedupBeforeTC},
        {"kT5Bin", (const void*)lst::kT5Bin},
        {"kT5DedupBinned", (const void*)lst::kT5DedupBinned},
        {"kMergeT5Flag", (const void*)lst::kMergeT5Flag},
        {"kCrossCleanT5", (const void*)lst::kCrossCleanT5},
        {"kT5TCCount", (const void*)lst::kT5TCCount},
        {"kT5TCScan", (const void*)lst::kT5TCScan},
        {"kT5TCEmit", (const void*)lst::kT5TCEmit},
        {"kT5TCFinish", (const void*)lst::kT5TCFinish},
        {"kTCCleanInfo", (const void*)lst::kTCCleanInfo},
        {"kCrossCleanPLS", (const void*)lst::kCrossCleanPLS},
        {"kAddPLSTC", (const void*)lst::kAddPLSTC},
        {"kCounts", (const void*)lst::kCounts},
        {"kSetInputCounts", (const void*)lst::kSetInputCounts},
        {"kUnpack", (const void*)lst::kUnpack},
        {"kOutputSizes", (const void*)lst::kOutputSizes},
        {"kOutputEventOffsets", (const void*)lst::kOutputEventOffsets},
        {"kOutputGather", (const void*)lst::kOutputGather},
    };
    return t;
  }

}  // namespace

extern "C" {

const char* lst_last_error(void) { return g_lastError.c_str(); }

int lst_kernel_count(void) {
  LST_ABI_TRY
  return static_cast<int>(kernelTable().size());
  LST_ABI_CATCH_INT
}

int lst_kernel_attributes(int i, const char** name, int* num_regs, int* max_threads_per_block, size_t* local_bytes,
                          size_t* static_smem_bytes) {
  LST_ABI_TRY
  const auto& t = kernelTable();
  if (i < 0 || i >= static_cast<int>(t.size()))
    return setError("kernel index out of range");
  cudaFuncAttributes a;
  LST_CUDA(cudaFuncGetAttributes(&a, t[i].fn));
  if (name)
    *name = t[i].name;
  if (num_regs)
    *num_regs = a.numRegs;
  if (max_threads_per_block)
    *max_threads_per_block = a.maxThreadsPerBlock;
  if (local_bytes)
    *local_bytes = a.localSizeBytes;
  if (static_smem_bytes)
    *static_smem_bytes = a.sharedSizeBytes;
  return 0;
  LST_ABI_CATCH_INT
}

int lst_es_load(const char* geometry_dir, const char* t5dnn_weights_path, int device, lst_es** out) {
  return lst_es_load_ex(geometry_dir, t5dnn_weights_path, device, 0u, out);
}

int lst_es_load_ex(const char* geometry_dir, const char* t5dnn_weights_path, int device, unsigned int flags,
                   lst_es** out) {
  LST_ABI_TRY
  if (!geometry_dir || !out)
    return setError("lst_es_load: null argument");
  *out = nullptr;
  if (flags & ~LST_ES_BUILD_ON_DEVICE)
    return setError("lst_es_load_ex: unknown flags");
  std::unique_ptr<lst_es> es(new (std::nothrow) lst_es());
  if (!es)
    return setError("out of host memory");
  es->device = device;
  // Every input file is read and checked before the first CUDA call: the
  // geometry, then the weights on the host path; the weights, then the
  // geometry (whose files the device build reads before its first CUDA
  // call) on the device path.
  const bool onDevice = (flags & LST_ES_BUILD_ON_DEVICE) != 0;
  if (!onDevice) {
    std::string err = lst::loadEsHost(geometry_dir, es->host);
    if (!err.empty())
      return setError(err);
  }
  if (t5dnn_weights_path) {
    int rc = loadWeightsFile(t5dnn_weights_path, es->dnn);
    if (rc)
      return rc;
  }
  if (onDevice) {
    std::string err = lst::buildEsOnDevice(geometry_dir, device, es->host);
    if (!err.empty())
      return setError(err);
  }
  for (int v : es->host.t5CapIfEligible)
    if (v >= 0)
      es->nEligibleMax++;
  LST_CUDA(cudaSetDevice(device));
  std::vector<std::pair<void*, const void*>> copies;
  std::vector<size_t> sizes;
  Carver measure;
  layoutES(measure, *es, copies, sizes);
  es->arenaBytes = measure.off;
  LST_CUDA(cudaMalloc(&es->arena, es->arenaBytes));
  Carver fill;
  fill.base = static_cast<char*>(es->arena);
  layoutES(fill, *es, copies, sizes);
  for (size_t i = 0; i < copies.size(); ++i)
    LST_CUDA(cudaMemcpy(copies[i].first, copies[i].second, sizes[i], cudaMemcpyHostToDevice));
  if (t5dnn_weights_path) {
    int rc = uploadWeights(es.get());
    if (rc) {
      cudaFree(es->arena);
      return rc;
    }
  }
  staticOutputDeviceRetain(device);
  *out = es.release();
  return 0;
  LST_ABI_CATCH_INT
}

int lst_es_load_host(const char* geometry_dir, lst_es** out) {
  LST_ABI_TRY
  if (!geometry_dir || !out)
    return setError("lst_es_load_host: null argument");
  *out = nullptr;
  std::unique_ptr<lst_es> es(new (std::nothrow) lst_es());
  if (!es)
    return setError("out of host memory");
  es->device = -1;
  std::string err = lst::loadEsHost(geometry_dir, es->host);
  if (!err.empty())
    return setError(err);
  *out = es.release();
  return 0;
  LST_ABI_CATCH_INT
}

int lst_es_host_array(const lst_es* es, const char* name, const void** data, size_t* n_elems, size_t* elem_size) {
  LST_ABI_TRY
  if (!es || !name || !data)
    return setError("lst_es_host_array: null argument");
  const lst::EsHost& h = es->host;
  const std::string key(name);
#define LST_ES_ARRAY(prefix, vec)                 \
  if (key == prefix #vec) {                       \
    *data = h.vec.data();                         \
    if (n_elems)                                  \
      *n_elems = h.vec.size();                    \
    if (elem_size)                                \
      *elem_size = sizeof(h.vec[0]);              \
    return 0;                                     \
  }
  LST_ES_ARRAY("modules.", detIds)
  LST_ES_ARRAY("modules.", moduleMap)
  LST_ES_ARRAY("modules.", mapdetId)
  LST_ES_ARRAY("modules.", mapIdx)
  LST_ES_ARRAY("modules.", nConnectedModules)
  LST_ES_ARRAY("modules.", drdzs)
  LST_ES_ARRAY("modules.", dxdys)
  LST_ES_ARRAY("modules.", partnerModuleIndices)
  LST_ES_ARRAY("modules.", layers)
  LST_ES_ARRAY("modules.", rings)
  LST_ES_ARRAY("modules.", modules)
  LST_ES_ARRAY("modules.", rods)
  LST_ES_ARRAY("modules.", subdets)
  LST_ES_ARRAY("modules.", sides)
  LST_ES_ARRAY("modules.", eta)
  LST_ES_ARRAY("modules.", r)
  LST_ES_ARRAY("modules.", isInverted)
  LST_ES_ARRAY("modules.", isLower)
  LST_ES_ARRAY("modules.", isAnchor)
  LST_ES_ARRAY("modules.", moduleType)
  LST_ES_ARRAY("modules.", moduleLayerType)
  LST_ES_ARRAY("modules.", sdlLayers)
  LST_ES_ARRAY("modules.", connectedPixels)
  LST_ES_ARRAY("pixelmap.", connectedPixelsIndex)
  LST_ES_ARRAY("pixelmap.", connectedPixelsSizes)
  LST_ES_ARRAY("pixelmap.", connectedPixelsIndexPos)
  LST_ES_ARRAY("pixelmap.", connectedPixelsSizesPos)
  LST_ES_ARRAY("pixelmap.", connectedPixelsIndexNeg)
  LST_ES_ARRAY("pixelmap.", connectedPixelsSizesNeg)
  LST_ES_ARRAY("endcap.", geoMapDetId)
  LST_ES_ARRAY("endcap.", geoMapPhi)
  LST_ES_ARRAY("endcap.", geoMapIndex)
  LST_ES_ARRAY("hash.", detHashKey)
  LST_ES_ARRAY("hash.", detHashVal)
  LST_ES_ARRAY("caps.", mdOffset)
  LST_ES_ARRAY("caps.", mdCap)
  LST_ES_ARRAY("caps.", lsOffset)
  LST_ES_ARRAY("caps.", lsCap)
  LST_ES_ARRAY("caps.", t3CapIfUsed)
  LST_ES_ARRAY("caps.", t5CapIfEligible)
#undef LST_ES_ARRAY
  return setError("unknown event-setup array " + key);
  LST_ABI_CATCH_INT
}

void lst_es_free(lst_es* es) {
  LST_ABI_TRY
  if (!es)
    return;
  if (es->arena) {
    cudaSetDevice(es->device);
    cudaFree(es->arena);
    staticOutputDeviceRelease(es->device);
  }
  delete es;
  LST_ABI_CATCH_VOID
}

int lst_es_get_info(const lst_es* es, lst_es_info* out) {
  LST_ABI_TRY
  if (!es || !out)
    return setError("lst_es_get_info: null argument");
  out->nModules = es->host.nModules;
  out->nLowerModules = es->host.nLowerModules;
  out->pixelModule = es->host.pixelModuleIndex;
  out->nConnectedPixels = es->host.nPixels;
  out->nTotalMDs = es->host.nTotalMDs;
  out->nTotalSegments = es->host.nTotalSegments;
  out->maxTriplets = es->host.maxTriplets;
  out->maxQuintuplets = es->host.maxQuintuplets;
  out->ptCut = es->host.ptCut;
  return 0;
  LST_ABI_CATCH_INT
}

int lst_es_set_t5dnn_weights(lst_es* es, const float* weights, size_t n) {
  LST_ABI_TRY
  if (!es || !weights)
    return setError("lst_es_set_t5dnn_weights: null argument");
  if (n != lst::kT5DnnParams)
    return setError("T5 DNN weights must hold 2337 values");
  es->dnn.assign(weights, weights + n);
  return uploadWeights(es);
  LST_ABI_CATCH_INT
}

int lst_event_create(lst_es* es, int n_slots, uint32_t max_hits, void* stream, lst_event** out) {
  LST_ABI_TRY
  if (!es || !out || n_slots <= 0 || max_hits == 0)
    return setError("lst_event_create: bad argument");
  if (es->device < 0 || !es->arena)
    return setError("lst_event_create: the event setup was loaded on the host only");
  *out = nullptr;
  std::unique_ptr<lst_event> ev(new (std::nothrow) lst_event());
  if (!ev)
    return setError("out of host memory");
  ev->es = es;
  ev->device = es->device;
  ev->nSlots = n_slots;
  ev->maxHits = max_hits;
  ev->t5Method = es->haveDnn ? LST_T5_DNN : LST_T5_CUTS;
  const lst::EsHost& h = es->host;
  ev->sizes = Sizes{max_hits,
                    h.nModules,
                    h.nLowerModules,
                    h.nTotalMDs,
                    h.nTotalSegments,
                    lst::kMaxPixelSegments,
                    std::max<size_t>(h.maxTriplets, 1),
                    std::max<size_t>(h.maxQuintuplets, 1),
                    lst::kMaxPixelTriplets,
                    lst::kMaxPixelQuintuplets,
                    lst::kMaxTrackCandidates};
  LST_CUDA(cudaSetDevice(es->device));
  LST_CUDA(cudaDeviceGetAttribute(&ev->nSM, cudaDevAttrMultiProcessorCount, es->device));
  for (int k = 0; k < kTuCount; ++k)
    ev->shape[k].warps = kTuneSpecs[k].defWarps;
  // Kernels whose shared memory exceeds the 48 KB default opt in (per device).
  LST_CUDA(cudaFuncSetAttribute(lst::kCrossCleanPLS, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(lst::kXCleanSmem)));
  LST_CUDA(cudaFuncSetAttribute(lst::kPT5DedupHashed, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(lst::kPT5DedupSmem)));
  LST_CUDA(cudaFuncSetAttribute(lst::kT5RankEmit, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(lst::kT5RankSmem)));
  Carver measure;
  lst::EventView tmp{};
  carveEvent(measure, tmp, ev->sizes);
  ev->slotBytes = (measure.off + 4095) & ~size_t(4095);
  ev->totalBytes = ev->slotBytes * n_slots;
  if (stream) {
    ev->stream = static_cast<cudaStream_t>(stream);
  } else {
    LST_CUDA(cudaStreamCreateWithFlags(&ev->stream, cudaStreamNonBlocking));
    ev->ownStream = true;
  }
  cudaError_t e = cudaMalloc(&ev->arena, ev->totalBytes);
  if (e != cudaSuccess) {
    if (ev->ownStream)
      cudaStreamDestroy(ev->stream);
    return cudaFail(e, "event arena");
  }
  LST_CUDA(cudaMalloc(&ev->dCounts, sizeof(lst_counts) * n_slots));
  ev->hv.resize(n_slots);
  for (int i = 0; i < n_slots; ++i) {
    Carver c;
    c.base = ev->arena + ev->slotBytes * i;
    carveEvent(c, ev->hv[i], ev->sizes);
    ev->hv[i].maxHits = max_hits;
    ev->hv[i].counts = ev->dCounts + i;
  }
  LST_CUDA(cudaMalloc(&ev->dv, sizeof(lst::EventView) * n_slots));
  LST_CUDA(cudaMemcpy(ev->dv, ev->hv.data(), sizeof(lst::EventView) * n_slots, cudaMemcpyHostToDevice));
  LST_CUDA(cudaMalloc(&ev->ownOffsets, sizeof(unsigned long long) * n_slots));
  ev->dOffsets = ev->ownOffsets;
  LST_CUDA(cudaMallocHost(&ev->hCounts, sizeof(lst_counts) * n_slots));
  LST_CUDA(cudaMalloc(&ev->dOutOffsets, sizeof(unsigned long long) * 2 * (n_slots + 1)));
  LST_CUDA(cudaMallocHost(&ev->hOutOffsets, sizeof(unsigned long long) * 2 * (n_slots + 1)));
  // Start every slot empty.
  int rc = runReset(ev.get(), 0, n_slots);
  if (rc)
    return rc;
  LST_CUDA(cudaStreamSynchronize(ev->stream));
  *out = ev.release();
  return 0;
  LST_ABI_CATCH_INT
}

void lst_event_destroy(lst_event* ev) {
  LST_ABI_TRY
  if (!ev)
    return;
  cudaSetDevice(ev->device);
  cudaStreamSynchronize(ev->stream);
  cudaFree(ev->arena);
  cudaFree(ev->dv);
  cudaFree(ev->ownOffsets);
  cudaFree(ev->dCounts);
  if (ev->ownInbox)
    cudaFree(ev->ownInbox);
  for (auto& b : ev->stage) {
    if (b.ptr)
      cudaFree(b.ptr);
    if (b.offsets)
      cudaFree(b.offsets);
    if (b.ready)
      cudaEventDestroy(b.ready);
    if (b.freed)
      cudaEventDestroy(b.freed);
  }
  if (ev->copyStream)
    cudaStreamDestroy(ev->copyStream);
  cudaFreeHost(ev->hCounts);
  cudaFree(ev->dOutOffsets);
  cudaFreeHost(ev->hOutOffsets);
  for (cudaEvent_t e : ev->eventPool)
    cudaEventDestroy(e);
  for (auto& g : ev->graphs)
    cudaGraphExecDestroy(g.second.exec);
  if (ev->dProbeCount)
    cudaFree(ev->dProbeCount);
  if (ev->dOut)
    cudaFree(ev->dOut);
  if (ev->ownStream)
    cudaStreamDestroy(ev->stream);
  delete ev;
  LST_ABI_CATCH_VOID
}

int lst_event_memory(const lst_event* ev, size_t* bytes) {
  LST_ABI_TRY
  if (!ev || !bytes)
    return setError("lst_event_memory: null argument");
  *bytes = ev->totalBytes + ev->inboxBytes + ev->stage[0].bytes + ev->stage[1].bytes;
  return 0;
  LST_ABI_CATCH_INT
}

int lst_event_sync(lst_event* ev) {
  LST_ABI_TRY
  if (!ev)
    return setError("null event set");
  LST_CUDA(cudaStreamSynchronize(ev->stream));
  return 0;
  LST_ABI_CATCH_INT
}

void* lst_event_stream(lst_event* ev) { return ev ? static_cast<void*>(ev->stream) : nullptr; }

int lst_event_set_t5_method(lst_event* ev, int method) {
  LST_ABI_TRY
  if (!ev)
    return setError("null event set");
  if (method != LST_T5_DNN && method != LST_T5_CUTS)
    return setError("unknown T5 method");
  if (method == LST_T5_DNN && !ev->es->haveDnn)
    return setError("the DNN T5 method needs weights");
  ev->t5Method = method;
  return 0;
  LST_ABI_CATCH_INT
}

int lst_event_set_walk(lst_event* ev, int on) {
  LST_ABI_TRY
  if (!ev)
    return setError("null event set");
  LST_CUDA(cudaStreamSynchronize(ev->stream));
  for (auto& v : ev->hv)
    v.forceWalk = on ? 1u : 0u;
  LST_CUDA(cudaMemcpy(ev->dv, ev->hv.data(), sizeof(lst::EventView) * ev->nSlots, cudaMemcpyHostToDevice));
  return 0;
  LST_ABI_CATCH_INT
}

int lst_event_reset(lst_event* ev, int slot) {
  LST_ABI_TRY
  int rc = checkSlots(ev, slot, 1);
  if (rc)
    return rc;
  return runReset(ev, slot, 1);
  LST_ABI_CATCH_INT
}

int lst_event_add_hits(lst_event* ev, int slot, uint32_t n, const float* x, const float* y, const float* z,
                       const uint32_t* detId, const uint32_t* idxInNtuple) {
  LST_ABI_TRY
  int rc = checkSlots(ev, slot, 1);
  if (rc)
    return rc;
  if (n > ev->maxHits)
    return LST_STATUS_HIT_CAPACITY;
  if (n > 0 && (!x || !y || !z || !detId || !idxInNtuple))
    return setError("lst_event_add_hits: null array");
  rc = runReset(ev, slot, 1);
  if (rc)
    return rc;
  const lst::EventView& v = ev->hv[slot];
  cudaStream_t s = ev->stream;
  if (n > 0) {
    LST_CUDA(cudaMemcpyAsync(v.hits.xs, x, n * sizeof(float), cudaMemcpyDefault, s));
    LST_CUDA(cudaMemcpyAsync(v.hits.ys, y, n * sizeof(float), cudaMemcpyDefault, s));
    LST_CUDA(cudaMemcpyAsync(v.hits.zs, z, n * sizeof(float), cudaMemcpyDefault, s));
    LST_CUDA(cudaMemcpyAsync(v.hits.detid, detId, n * sizeof(uint32_t), cudaMemcpyDefault, s));
    LST_CUDA(cudaMemcpyAsync(v.hits.idxs, idxInNtuple, n * sizeof(uint32_t), cudaMemcpyDefault, s));
  }
  LST_LAUNCH(lst::kSetInputCounts, 1, 1, ev->dv, slot, 1, n, 1, 0u, 0u);
  return runHitKernels(ev, slot, 1);
  LST_ABI_CATCH_INT
}

int lst_event_add_pixel_segments(lst_event* ev, int slot, uint32_t n, const uint32_t* hitIndices0,
                                 const uint32_t* hitIndices1, const uint32_t* hitIndices2,
                                 const uint32_t* hitIndices3, const float* dPhiChange, const float* ptIn,
                                 const float* ptErr, const float* px, const float* py, const float* pz,
                                 const float* eta, const float* etaErr, const float* phi, const int32_t* charge,
                                 const uint32_t* seedIdx, const int32_t* superbin, const int8_t* pixelType,
                                 const int8_t* isQuad) {
  LST_ABI_TRY
  int rc = checkSlots(ev, slot, 1);
  if (rc)
    return rc;
  unsigned int status = 0;
  uint32_t size = n;
  if (size > lst::kMaxPixelSegments) {
    size = lst::kMaxPixelSegments;
    status |= LST_STATUS_PLS_TRUNCATED;
  }
  if (size > 0 && (!hitIndices0 || !hitIndices1 || !hitIndices2 || !hitIndices3 || !dPhiChange || !ptIn || !ptErr ||
                   !px || !py || !pz || !eta || !etaErr || !phi || !charge || !seedIdx || !superbin || !pixelType ||
                   !isQuad))
    return setError("lst_event_add_pixel_segments: null array");
  const lst::EventView& v = ev->hv[slot];
  cudaStream_t s = ev->stream;
  if (size > 0) {
    LST_CUDA(cudaMemcpyAsync(v.plsHit0, hitIndices0, size * 4, cudaMemcpyDefault, s));
    LST_CUDA(cudaMemcpyAsync(v.plsHit1, hitIndices1, size * 4, cudaMemcpyDefault, s));
    LST_CUDA(cudaMemcpyAsync(v.plsHit2, hitIndices2, size * 4, cudaMemcpyDefault, s));
    LST_CUDA(cudaMemcpyAsync(v.plsHit3, hitIndices3, size * 4, cudaMemcpyDefault, s));
    LST_CUDA(cudaMemcpyAsync(v.plsDPhiChange, dPhiChange, size * 4, cudaMemcpyDefault, s));
    LST_CUDA(cudaMemcpyAsync(v.ls.ptIn, ptIn, size * 4, cudaMemcpyDefault, s));
    LST_CUDA(cudaMemcpyAsync(v.ls.ptErr, ptErr, size * 4, cudaMemcpyDefault, s));
    LST_CUDA(cudaMemcpyAsync(v.ls.px, px, size * 4, cudaMemcpyDefault, s));
    LST_CUDA(cudaMemcpyAsync(v.ls.py, py, size * 4, cudaMemcpyDefault, s));
    LST_CUDA(cudaMemcpyAsync(v.ls.pz, pz, size * 4, cudaMemcpyDefault, s));
    LST_CUDA(cudaMemcpyAsync(v.ls.etaErr, etaErr, size * 4, cudaMemcpyDefault, s));
    LST_CUDA(cudaMemcpyAsync(v.ls.isQuad, isQuad, size, cudaMemcpyDefault, s));
    LST_CUDA(cudaMemcpyAsync(v.ls.eta, eta, size * 4, cudaMemcpyDefault, s));
    LST_CUDA(cudaMemcpyAsync(v.ls.phi, phi, size * 4, cudaMemcpyDefault, s));
    LST_CUDA(cudaMemcpyAsync(v.ls.charge, charge, size * 4, cudaMemcpyDefault, s));
    LST_CUDA(cudaMemcpyAsync(v.ls.seedIdx, seedIdx, size * 4, cudaMemcpyDefault, s));
    LST_CUDA(cudaMemcpyAsync(v.ls.superbin, superbin, size * 4, cudaMemcpyDefault, s));
    LST_CUDA(cudaMemcpyAsync(v.ls.pixelType, pixelType, size, cudaMemcpyDefault, s));
  }
  LST_LAUNCH(lst::kSetInputCounts, 1, 1, ev->dv, slot, 0, 0u, 1, size, status);
  return runPixelIngest(ev, slot, 1);
  LST_ABI_CATCH_INT
}

int lst_event_run_stage(lst_event* ev, int slot, int stage) {
  LST_ABI_TRY
  int rc = checkSlots(ev, slot, 1);
  if (rc)
    return rc;
  return runStage(ev, slot, 1, stage);
  LST_ABI_CATCH_INT
}

int lst_event_create_mini_doublets(lst_event* ev, int slot) {
  LST_ABI_TRY
  return lst_event_run_stage(ev, slot, LST_STAGE_MINI_DOUBLETS);
  LST_ABI_CATCH_INT
}
int lst_event_create_segments(lst_event* ev, int slot) {
  LST_ABI_TRY
  return lst_event_run_stage(ev, slot, LST_STAGE_SEGMENTS);
  LST_ABI_CATCH_INT
}
int lst_event_create_triplets(lst_event* ev, int slot) {
  LST_ABI_TRY
  return lst_event_run_stage(ev, slot, LST_STAGE_TRIPLETS);
  LST_ABI_CATCH_INT
}
int lst_event_create_quintuplets(lst_event* ev, int slot) {
  LST_ABI_TRY
  return lst_event_run_stage(ev, slot, LST_STAGE_QUINTUPLETS);
  LST_ABI_CATCH_INT
}
int lst_event_pixel_line_segment_cleaning(lst_event* ev, int slot) {
  LST_ABI_TRY
  return lst_event_run_stage(ev, slot, LST_STAGE_PLS_CLEANING);
  LST_ABI_CATCH_INT
}
int lst_event_create_pixel_quintuplets(lst_event* ev, int slot) {
  LST_ABI_TRY
  return lst_event_run_stage(ev, slot, LST_STAGE_PIXEL_QUINTUPLETS);
  LST_ABI_CATCH_INT
}
int lst_event_create_pixel_triplets(lst_event* ev, int slot) {
  LST_ABI_TRY
  return lst_event_run_stage(ev, slot, LST_STAGE_PIXEL_TRIPLETS);
  LST_ABI_CATCH_INT
}
int lst_event_create_track_candidates(lst_event* ev, int slot) {
  LST_ABI_TRY
  return lst_event_run_stage(ev, slot, LST_STAGE_TRACK_CANDIDATES);
  LST_ABI_CATCH_INT
}

int lst_event_get_counts(lst_event* ev, int slot, lst_counts* out) {
  LST_ABI_TRY
  int rc = checkSlots(ev, slot, 1);
  if (rc)
    return rc;
  if (!out)
    return setError("lst_event_get_counts: null output");
  rc = readCounts(ev, slot, 1, out);
  if (rc)
    return rc;
  return static_cast<int>(out->status & 0x7fffffffu);
  LST_ABI_CATCH_INT
}

int lst_event_get_field(lst_event* ev, int slot, const char* name, void* dst, size_t capacity, size_t* n_elems,
                        size_t* elem_size) {
  LST_ABI_TRY
  int rc = checkSlots(ev, slot, 1);
  if (rc)
    return rc;
  if (!name)
    return setError("lst_event_get_field: null name");
  void* ptr = nullptr;
  size_t n = 0, esz = 0;
  if (!findField(ev->hv[slot], ev->sizes, name, ptr, n, esz))
    return setError(std::string("unknown field ") + name);
  if (n_elems)
    *n_elems = n;
  if (elem_size)
    *elem_size = esz;
  if (dst && capacity) {
    size_t k = std::min(n, capacity);
    LST_CUDA(cudaMemcpyAsync(dst, ptr, k * esz, cudaMemcpyDeviceToHost, ev->stream));
    LST_CUDA(cudaStreamSynchronize(ev->stream));
  }
  return 0;
  LST_ABI_CATCH_INT
}

int lst_event_field_device_ptr(lst_event* ev, int slot, const char* name, void** dptr, size_t* n_elems,
                               size_t* elem_size) {
  LST_ABI_TRY
  int rc = checkSlots(ev, slot, 1);
  if (rc)
    return rc;
  if (!name || !dptr)
    return setError("lst_event_field_device_ptr: null argument");
  size_t n = 0, esz = 0;
  if (!findField(ev->hv[slot], ev->sizes, name, *dptr, n, esz))
    return setError(std::string("unknown field ") + name);
  if (n_elems)
    *n_elems = n;
  if (elem_size)
    *elem_size = esz;
  return 0;
  LST_ABI_CATCH_INT
}

int lst_field_count(void) {
  LST_ABI_TRY
  return static_cast<int>(fieldTable().size());
  LST_ABI_CATCH_INT
}

const char* lst_field_name(int i) {
  try {
    const auto& t = fieldTable();
    if (i < 0 || i >= static_cast<int>(t.size()))
      return nullptr;
    return t[i].name.c_str();
  } catch (...) {
    return nullptr;
  }
}

int lst_field_info(int i, const char** name, size_t* elem_size, char* kind) {
  LST_ABI_TRY
  const auto& t = fieldTable();
  if (i < 0 || i >= static_cast<int>(t.size()))
    return setError("field index out of range");
  if (name)
    *name = t[i].name.c_str();
  if (elem_size)
    *elem_size = t[i].elemSize;
  if (kind)
    *kind = t[i].kind;
  return 0;
  LST_ABI_CATCH_INT
}

size_t lst_packed_size(uint32_t n_hits, uint32_t n_pls) { return lst::packedLayout(n_hits, n_pls).end; }

namespace {
  // Copies packed events into the set's device inbox and ingests them.
  int uploadInbox(lst_event* ev, int first, int count, const void* blobs, size_t total_bytes,
                  const uint64_t* blob_offsets, int kind, const char* who) {
    int rc = checkSlots(ev, first, count);
    if (rc)
      return rc;
    if (count == 0)
      return 0;
    if (!blobs || !blob_offsets)
      return setError(std::string(who) + ": null argument");
    for (int i = 0; i < count; ++i) {
      if (blob_offsets[i] % 16 != 0 || blob_offsets[i] + 16 > total_bytes)
        return setError(std::string(who) + ": blob offset misaligned or outside the buffer");
    }
    if (total_bytes > ev->inboxBytes) {
    LST_CUDA(cudaStreamSynchronize(ev->stream));
    if (ev->ownInbox)
      LST_CUDA(cudaFree(ev->ownInbox));
    ev->ownInbox = nullptr;
    ev->inboxBytes = 0;
    size_t want = (total_bytes + (1u << 20) - 1) & ~size_t((1u << 20) - 1);
    LST_CUDA(cudaMalloc(&ev->ownInbox, want));
    ev->inboxBytes = want;
  }
  cudaStream_t s = ev->stream;
  LST_CUDA(cudaMemcpyAsync(ev->ownInbox, blobs, total_bytes, cudaMemcpyDefault, s));
  LST_CUDA(cudaMemcpyAsync(ev->ownOffsets + first, blob_offsets, sizeof(uint64_t) * count, cudaMemcpyDefault, s));
  ev->inbox = ev->ownInbox;
  ev->dOffsets = ev->ownOffsets;
  ev->inboxValid = true;
  ev->inboxUsed = total_bytes;
  ev->inboxKind = kind;
  ev->inboxFirst = first;
  ev->inboxCount = count;
  return ingestInbox(ev, first, count);
  }
}  // namespace

int lst_batch_upload(lst_event* ev, int first, int count, const void* blobs, size_t total_bytes,
                     const uint64_t* blob_offsets) {
  LST_ABI_TRY
  return uploadInbox(ev, first, count, blobs, total_bytes, blob_offsets, 0, "lst_batch_upload");
  LST_ABI_CATCH_INT
}

int lst_batch_upload_seeds(lst_event* ev, int first, int count, const void* blobs, size_t total_bytes,
                           const uint64_t* blob_offsets) {
  LST_ABI_TRY
  return uploadInbox(ev, first, count, blobs, total_bytes, blob_offsets, 1, "lst_batch_upload_seeds");
  LST_ABI_CATCH_INT
}

int lst_batch_stage(lst_event* ev, int first, int count, const void* blobs, size_t total_bytes,
                    const uint64_t* blob_offsets, int seed_layout) {
  LST_ABI_TRY
  int rc = checkSlots(ev, first, count);
  if (rc)
    return rc;
  if (count == 0)
    return setError("lst_batch_stage: no slots");
  if (!blobs || !blob_offsets)
    return setError("lst_batch_stage: null argument");
  for (int i = 0; i < count; ++i)
    if (blob_offsets[i] % 16 != 0 || blob_offsets[i] + 16 > total_bytes)
      return setError("lst_batch_stage: blob offset misaligned or outside the buffer");
  if (ev->staged.pending)
    return setError("lst_batch_stage: a staged batch has not been ingested yet");
  if (!ev->copyStream)
    LST_CUDA(cudaStreamCreateWithFlags(&ev->copyStream, cudaStreamNonBlocking));
  lst_event::StageBuf& b = ev->stage[ev->stageNext];
  if (!b.ready) {
    LST_CUDA(cudaEventCreateWithFlags(&b.ready, cudaEventDisableTiming));
    LST_CUDA(cudaEventCreateWithFlags(&b.freed, cudaEventDisableTiming));
    LST_CUDA(cudaMalloc(&b.offsets, sizeof(unsigned long long) * ev->nSlots));
  }
  if (total_bytes > b.bytes) {
    // the buffer may still be read by an ingest or written by a copy
    LST_CUDA(cudaStreamSynchronize(ev->stream));
    LST_CUDA(cudaStreamSynchronize(ev->copyStream));
    if (b.ptr)
      LST_CUDA(cudaFree(b.ptr));
    b.ptr = nullptr;
    b.bytes = 0;
    const size_t want = (total_bytes + (1u << 20) - 1) & ~size_t((1u << 20) - 1);
    LST_CUDA(cudaMalloc(&b.ptr, want));
    b.bytes = want;
    LST_CUDA(cudaEventRecord(b.freed, ev->stream));
  }
  LST_CUDA(cudaStreamWaitEvent(ev->copyStream, b.freed, 0));
  LST_CUDA(cudaMemcpyAsync(b.ptr, blobs, total_bytes, cudaMemcpyDefault, ev->copyStream));
  LST_CUDA(cudaMemcpyAsync(b.offsets + first, blob_offsets, sizeof(uint64_t) * count, cudaMemcpyDefault,
                           ev->copyStream));
  LST_CUDA(cudaEventRecord(b.ready, ev->copyStream));
  ev->staged.pending = true;
  ev->staged.first = first;
  ev->staged.count = count;
  ev->staged.kind = seed_layout ? 1 : 0;
  ev->staged.buf = ev->stageNext;
  ev->staged.total = total_bytes;
  ev->stageNext ^= 1;
  return 0;
  LST_ABI_CATCH_INT
}

int lst_batch_ingest_staged(lst_event* ev) {
  LST_ABI_TRY
  if (!ev)
    return setError("null event set");
  if (!ev->staged.pending)
    return setError("lst_batch_ingest_staged: nothing staged");
  lst_event::StageBuf& b = ev->stage[ev->staged.buf];
  LST_CUDA(cudaStreamWaitEvent(ev->stream, b.ready, 0));
  ev->inbox = b.ptr;
  ev->dOffsets = b.offsets;
  ev->inboxValid = true;
  ev->inboxUsed = ev->staged.total;
  ev->inboxKind = ev->staged.kind;
  ev->inboxFirst = ev->staged.first;
  ev->inboxCount = ev->staged.count;
  ev->staged.pending = false;
  int rc = ingestInbox(ev, ev->staged.first, ev->staged.count);
  if (rc)
    return rc;
  LST_CUDA(cudaEventRecord(b.freed, ev->stream));
  return 0;
  LST_ABI_CATCH_INT
}

int lst_batch_ingest(lst_event* ev, int first, int count) {
  LST_ABI_TRY
  int rc = checkSlots(ev, first, count);
  if (rc)
    return rc;
  if (!ev->inboxValid)
    return setError("lst_batch_ingest: no packed inputs uploaded");
  if (count > 0 && (first < ev->inboxFirst || first + count > ev->inboxFirst + ev->inboxCount))
    return setError("lst_batch_ingest: slots outside the range of the last upload");
  if (count == 0)
    return 0;
  rc = ingestInbox(ev, first, count);
  if (rc)
    return rc;
  for (auto& b : ev->stage)  // a staging buffer being re-read must not be refilled before this ingest ends
    if (b.ptr && ev->inbox == b.ptr)
      LST_CUDA(cudaEventRecord(b.freed, ev->stream));
  return 0;
  LST_ABI_CATCH_INT
}

size_t lst_seed_packed_size(uint32_t n_ph2, uint32_t n_seeds, uint32_t n_seed_hits) {
  return lst::seedLayout(n_ph2, n_seeds, n_seed_hits).end;
}

int lst_seed_pack(const lst_seed_input* in, void* dst, size_t capacity) {
  LST_ABI_TRY
  if (!in || !dst)
    return setError("lst_seed_pack: null argument");
  const uint32_t nS = in->n_seeds, nH = in->n_ph2;
  const float* f[lst::kSeedFloatArrays] = {in->see_px,
                                           in->see_py,
                                           in->see_pz,
                                           in->see_dxy,
                                           in->see_dz,
                                           in->see_ptErr,
                                           in->see_etaErr,
                                           in->see_stateTrajGlbX,
                                           in->see_stateTrajGlbY,
                                           in->see_stateTrajGlbZ,
                                           in->see_stateTrajGlbPx,
                                           in->see_stateTrajGlbPy,
                                           in->see_stateTrajGlbPz};
  if (nS > 0) {
    for (const float* a : f)
      if (!a)
        return setError("lst_seed_pack: null seed array");
    if (!in->see_q || !in->see_hitIdx_offsets)
      return setError("lst_seed_pack: null seed array");
  }
  if (nH > 0 && (!in->ph2_detId || !in->ph2_x || !in->ph2_y || !in->ph2_z))
    return setError("lst_seed_pack: null hit array");
  const uint32_t* off = in->see_hitIdx_offsets;
  const uint32_t nSH = nS > 0 ? off[nS] : 0;
  if (nS > 0) {
    if (off[0] != 0)
      return setError("lst_seed_pack: see_hitIdx_offsets[0] must be 0");
    for (uint32_t i = 0; i < nS; ++i)
      if (off[i + 1] < off[i])
        return setError("lst_seed_pack: see_hitIdx_offsets not ascending at seed " + std::to_string(i));
    if (nSH > 0 && !in->see_hitIdx)
      return setError("lst_seed_pack: null see_hitIdx");
  }
  const lst::SeedLayout L = lst::seedLayout(nH, nS, nSH);
  if (capacity < L.end)
    return setError("lst_seed_pack: destination holds " + std::to_string(capacity) + " bytes, the event needs " +
                    std::to_string(L.end));
  unsigned char* d = static_cast<unsigned char*>(dst);
  const uint32_t hdr[4] = {nH, nS, nSH, lst::kSeedMagic};
  std::memcpy(d, hdr, sizeof(hdr));
  if (nH > 0) {
    std::memcpy(d + L.detId, in->ph2_detId, 4 * size_t(nH));
    std::memcpy(d + L.x, in->ph2_x, 4 * size_t(nH));
    std::memcpy(d + L.y, in->ph2_y, 4 * size_t(nH));
    std::memcpy(d + L.z, in->ph2_z, 4 * size_t(nH));
  }
  if (nS > 0) {
    for (int k = 0; k < lst::kSeedFloatArrays; ++k)
      std::memcpy(d + L.f[k], f[k], 4 * size_t(nS));
    std::memcpy(d + L.q, in->see_q, 4 * size_t(nS));
    std::memcpy(d + L.hitOff, off, 4 * (size_t(nS) + 1));
    if (nSH > 0)
      std::memcpy(d + L.hitIdx, in->see_hitIdx, 4 * size_t(nSH));
  } else {
    std::memset(d + L.hitOff, 0, 4);
  }
  if (L.end > L.hitIdx + 4 * size_t(nSH))
    std::memset(d + L.hitIdx + 4 * size_t(nSH), 0, L.end - L.hitIdx - 4 * size_t(nSH));
  return 0;
  LST_ABI_CATCH_INT
}

int lst_event_prepare_input(lst_event* ev, int slot, const lst_seed_input* in) {
  LST_ABI_TRY
  int rc = checkSlots(ev, slot, 1);
  if (rc)
    return rc;
  if (!in)
    return setError("lst_event_prepare_input: null input");
  const uint32_t nSH = in->n_seeds > 0 && in->see_hitIdx_offsets ? in->see_hitIdx_offsets[in->n_seeds] : 0;
  const size_t need = lst_seed_packed_size(in->n_ph2, in->n_seeds, nSH);
  // Pageable staging: cudaMemcpyAsync from pageable memory returns once the
  // bytes are taken, so the vector can be refilled by the next call.
  if (ev->hostPack.size() < need)
    ev->hostPack.resize(need);
  rc = lst_seed_pack(in, ev->hostPack.data(), ev->hostPack.size());
  if (rc)
    return rc;
  const uint64_t offset = 0;
  return lst_batch_upload_seeds(ev, slot, 1, ev->hostPack.data(), need, &offset);
  LST_ABI_CATCH_INT
}

int lst_run(lst_event* ev, int slot, const lst_seed_input* in, lst_output* out) {
  LST_ABI_TRY
  int rc = lst_event_prepare_input(ev, slot, in);
  if (rc)
    return rc;
  rc = lst_batch_run(ev, slot, 1, LST_STAGE_MINI_DOUBLETS, LST_STAGE_TRACK_CANDIDATES);
  if (rc)
    return rc;
  return out ? lst_batch_get_output(ev, slot, 1, out) : 0;
  LST_ABI_CATCH_INT
}

int lst_batch_run(lst_event* ev, int first, int count, int first_stage, int last_stage) {
  LST_ABI_TRY
  int rc = checkSlots(ev, first, count);
  if (rc)
    return rc;
  if (count == 0)
    return 0;
  if (first_stage < LST_STAGE_MINI_DOUBLETS || last_stage > LST_STAGE_TRACK_CANDIDATES || first_stage > last_stage)
    return setError("lst_batch_run: bad stage range");
  // Stage order of a full event (SDL/LST.cc:34-81): the pT5 stage runs
  // before the pT3 stage.
  static const int order[] = {LST_STAGE_MINI_DOUBLETS,
                              LST_STAGE_SEGMENTS,
                              LST_STAGE_TRIPLETS,
                              LST_STAGE_QUINTUPLETS,
                              LST_STAGE_PLS_CLEANING,
                              LST_STAGE_PIXEL_QUINTUPLETS,
                              LST_STAGE_PIXEL_TRIPLETS,
                              LST_STAGE_TRACK_CANDIDATES};
  for (int st : order) {
    if (st < first_stage || st > last_stage)
      continue;
    rc = runStage(ev, first, count, st);
    if (rc)
      return rc;
  }
  return 0;
  LST_ABI_CATCH_INT
}

int lst_batch_run_graph(lst_event* ev, int first, int count, int first_stage, int last_stage) {
  LST_ABI_TRY
  int rc = checkSlots(ev, first, count);
  if (rc)
    return rc;
  if (count == 0)
    return 0;
  if (ev->profiling)  // timing events cannot be read back from graph replays
    return lst_batch_run(ev, first, count, first_stage, last_stage);
  const auto key = std::make_tuple(first, count, first_stage, last_stage, ev->t5Method, ev->hv[first].forceWalk);
  auto it = ev->graphs.find(key);
  if (it == ev->graphs.end()) {
    cudaGraph_t graph = nullptr;
    LST_CUDA(cudaStreamBeginCapture(ev->stream, cudaStreamCaptureModeThreadLocal));
    const unsigned long long before = ev->launches;
    rc = lst_batch_run(ev, first, count, first_stage, last_stage);
    cudaError_t e = cudaStreamEndCapture(ev->stream, &graph);
    if (rc)
      return rc;
    if (e != cudaSuccess)
      return cudaFail(e, "cudaStreamEndCapture");
    lst_event::GraphEntry entry;
    entry.kernels = ev->launches - before;
    ev->launches = before;
    e = cudaGraphInstantiate(&entry.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess)
      return cudaFail(e, "cudaGraphInstantiate");
    it = ev->graphs.emplace(key, entry).first;
  }
  LST_CUDA(cudaGraphLaunch(it->second.exec, ev->stream));
  ev->launches += it->second.kernels;
  return 0;
  LST_ABI_CATCH_INT
}

int lst_batch_t5_probe(lst_event* ev, int first, int count, float* feat, float* score, uint8_t* cut_pass,
                       uint8_t* rz_tight, uint32_t* hits, int32_t* event_index, uint32_t capacity,
                       uint32_t* n_found) {
  LST_ABI_TRY
  int rc = checkSlots(ev, first, count);
  if (rc)
    return rc;
  if (!n_found || (capacity && (!feat || !score || !cut_pass || !rz_tight || !hits || !event_index)))
    return setError("lst_batch_t5_probe: null argument");
  if (!ev->es->haveDnn)
    return setError("lst_batch_t5_probe: needs T5 DNN weights");
  *n_found = 0;
  if (count == 0)
    return 0;
  if (!ev->dProbeCount)
    LST_CUDA(cudaMalloc(&ev->dProbeCount, sizeof(unsigned int)));
  cudaStream_t s = ev->stream;
  const lst::DeviceES& d = ev->es->view;
  const lst::EventView* v = ev->dv + first;
  LST_CUDA(cudaMemsetAsync(ev->dProbeCount, 0, sizeof(unsigned int), s));
  LST_LAUNCH(lst::kT5Prefix, warpGrid(ev->es->nEligibleMax, 8, count), 256, d, v);
  LST_LAUNCH(lst::kT5ModScan, dim3(1, count), 1024, d, v);
  lst::T5ProbeOut out{feat, score, cut_pass, rz_tight, hits, event_index, capacity, ev->dProbeCount};
  LST_LAUNCH(lst::kT5Probe, dim3(2 * kResidentBlocks / std::max(count, 1) + 1, count), 128, d, v, first, out);
  unsigned int n = 0;
  LST_CUDA(cudaMemcpyAsync(&n, ev->dProbeCount, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
  LST_CUDA(cudaStreamSynchronize(s));
  *n_found = n;
  return 0;
  LST_ABI_CATCH_INT
}

int lst_es_set_t5dnn_threshold(lst_es* es, float wp) {
  LST_ABI_TRY
  if (!es || es->device < 0)
    return setError("lst_es_set_t5dnn_threshold: no device event setup");
  LST_CUDA(cudaSetDevice(es->device));
  LST_CUDA(cudaMemcpyToSymbol(lst::c_t5dnnWP, &wp, sizeof(float)));
  LST_CUDA(cudaDeviceSynchronize());
  return 0;
  LST_ABI_CATCH_INT
}

int lst_batch_get_counts(lst_event* ev, int first, int count, lst_counts* out) {
  LST_ABI_TRY
  int rc = checkSlots(ev, first, count);
  if (rc)
    return rc;
  if (!out)
    return setError("lst_batch_get_counts: null output");
  if (count == 0)
    return 0;
  return readCounts(ev, first, count, out);
  LST_ABI_CATCH_INT
}

int lst_batch_get_output(lst_event* ev, int first, int count, lst_output* out) {
  LST_ABI_TRY
  int rc = checkSlots(ev, first, count);
  if (rc)
    return rc;
  if (!out || !out->event_tc_offsets || !out->event_hit_offsets)
    return setError("lst_batch_get_output: null output");
  if (count == 0) {
    out->event_tc_offsets[0] = 0;
    out->event_hit_offsets[0] = 0;
    return 0;
  }
  cudaStream_t s = ev->stream;
  const lst::EventView* v = ev->dv + first;
  LST_LAUNCH(lst::kOutputSizes, dim3(1, count), 1024, v);
  LST_LAUNCH(lst::kOutputEventOffsets, 1, 1024, v, count, ev->dOutOffsets);
  const size_t nOff = 2 * (size_t(count) + 1);
  LST_CUDA(cudaMemcpyAsync(ev->hOutOffsets, ev->dOutOffsets, sizeof(unsigned long long) * nOff,
                           cudaMemcpyDeviceToHost, s));
  LST_CUDA(cudaStreamSynchronize(s));
  const unsigned long long* tcOff = ev->hOutOffsets;
  const unsigned long long* hitOff = ev->hOutOffsets + count + 1;
  for (int i = 0; i <= count; ++i) {
    out->event_tc_offsets[i] = tcOff[i];
    out->event_hit_offsets[i] = hitOff[i];
  }
  const size_t nTC = tcOff[count], nHits = hitOff[count];
  if (nTC > out->tc_capacity || nHits > out->hits_capacity)
    return setError("lst_batch_get_output: output capacity too small (" + std::to_string(nTC) + " candidates, " +
                    std::to_string(nHits) + " hits needed)");
  if (nTC == 0)
    return 0;
  if (!out->hits || !out->len || !out->seedIdx || !out->type)
    return setError("lst_batch_get_output: null output array");
  // Device staging: hits | len | seedIdx | type, each 256-byte aligned.
  Carver c;
  c.take<unsigned int>(nHits);
  c.take<unsigned int>(nTC);
  c.take<int>(nTC);
  c.take<short>(nTC);
  if (c.off > ev->dOutBytes) {
    if (ev->dOut)
      LST_CUDA(cudaFree(ev->dOut));
    ev->dOut = nullptr;
    ev->dOutBytes = 0;
    size_t want = (c.off + (4u << 20) - 1) & ~size_t((4u << 20) - 1);
    LST_CUDA(cudaMalloc(&ev->dOut, want));
    ev->dOutBytes = want;
  }
  Carver d;
  d.base = reinterpret_cast<char*>(ev->dOut);
  unsigned int* dHits = d.take<unsigned int>(nHits);
  unsigned int* dLen = d.take<unsigned int>(nTC);
  int* dSeed = d.take<int>(nTC);
  short* dType = d.take<short>(nTC);
  LST_LAUNCH(lst::kOutputGather, dim3(blocksFor(lst::kMaxTrackCandidates, count), count), kThreads, v, count,
             ev->dOutOffsets, dHits, dLen, dSeed, dType);
  LST_CUDA(cudaMemcpyAsync(out->hits, dHits, nHits * sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
  LST_CUDA(cudaMemcpyAsync(out->len, dLen, nTC * sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
  LST_CUDA(cudaMemcpyAsync(out->seedIdx, dSeed, nTC * sizeof(int), cudaMemcpyDeviceToHost, s));
  LST_CUDA(cudaMemcpyAsync(out->type, dType, nTC * sizeof(short), cudaMemcpyDeviceToHost, s));
  LST_CUDA(cudaStreamSynchronize(s));
  return 0;
  LST_ABI_CATCH_INT
}

}  // extern "C"

// ------------------------------------------- output without device allocation
// lst_batch_get_output stages the flattened track-candidate output in a device
// buffer that it grows with cudaMalloc when a batch needs more room.  Some
// callers cannot allocate at that point: a framework whose caching allocator
// owns the device memory budget, or a producer that must not call cudaFree /
// cudaMalloc between events because those calls synchronise the whole device
// and stall the other streams.  lst_batch_get_output_static does the same work
// with its staging in a fixed, file-scope device array instead.
namespace {

  // Bytes of the static staging array, and the part of it that holds the
  // per-event offsets (2 x (events + 1) x 8 bytes).
  constexpr size_t kStaticOutputBytes = size_t(4) << 20;
  constexpr size_t kStaticOffsetBytes = size_t(16) << 10;
  constexpr int kStaticOutputMaxEvents = static_cast<int>(kStaticOffsetBytes / (2 * sizeof(unsigned long long))) - 1;

  static __device__ __align__(256) unsigned char g_staticOutput[kStaticOutputBytes];

  // Device address of g_staticOutput per device, looked up once per device
  // with that device current.  The address is cached only while an event
  // setup is alive on the device: freeing the last one forgets it, so a
  // device reset between two event setups cannot leave a stale address.  (A
  // cudaDeviceReset while an event setup is still alive invalidates that
  // event setup and its event sets as well, and is not supported.)
  constexpr int kMaxDevices = 64;
  std::mutex g_staticOutputMutex;
  unsigned char* g_staticOutputPtr[kMaxDevices] = {};
  int g_liveEsPerDevice[kMaxDevices] = {};

  void staticOutputDeviceRetain(int device) {
    if (device < 0 || device >= kMaxDevices)
      return;
    std::lock_guard<std::mutex> lock(g_staticOutputMutex);
    ++g_liveEsPerDevice[device];
  }

  void staticOutputDeviceRelease(int device) {
    if (device < 0 || device >= kMaxDevices)
      return;
    std::lock_guard<std::mutex> lock(g_staticOutputMutex);
    if (g_liveEsPerDevice[device] > 0 && --g_liveEsPerDevice[device] == 0)
      g_staticOutputPtr[device] = nullptr;
  }

  int staticOutputScratch(int device, unsigned char** out) {
    if (device < 0 || device >= kMaxDevices)
      return setError("device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_staticOutputMutex);
    if (!g_staticOutputPtr[device]) {
      int current = 0;
      LST_CUDA(cudaGetDevice(&current));
      if (current != device)
        LST_CUDA(cudaSetDevice(device));
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_staticOutput);
      if (current != device)
        cudaSetDevice(current);
      if (e != cudaSuccess)
        return cudaFail(e, "cudaGetSymbolAddress(static output staging)");
      g_staticOutputPtr[device] = static_cast<unsigned char*>(p);
    }
    *out = g_staticOutputPtr[device];
    return 0;
  }

  // Launch without the profiling hook (which creates CUDA events on demand).
#define LST_LAUNCH_PLAIN(kernel, grid, block, ...)             \
  do {                                                         \
    cudaGetLastError(); /* drop a stale non-sticky error */    \
    kernel<<<(grid), (block), 0, s>>>(__VA_ARGS__);            \
    cudaError_t e_ = cudaGetLastError();                       \
    if (e_ != cudaSuccess)                                     \
      return cudaFail(e_, #kernel);                            \
    ++ev->launches;                                            \
  } while (0)

}  // namespace

extern "C" {

int lst_batch_get_output_static(lst_event* ev, int first, int count, lst_output* out) {
  LST_ABI_TRY
  int rc = checkSlots(ev, first, count);
  if (rc)
    return rc;
  if (!out || !out->event_tc_offsets || !out->event_hit_offsets)
    return setError("lst_batch_get_output_static: null output");
  if (count == 0) {
    out->event_tc_offsets[0] = 0;
    out->event_hit_offsets[0] = 0;
    return 0;
  }
  if (count > kStaticOutputMaxEvents)
    return setError("lst_batch_get_output_static: at most " + std::to_string(kStaticOutputMaxEvents) +
                    " events per call (split the slot range)");
  unsigned char* scratch = nullptr;
  rc = staticOutputScratch(ev->es->device, &scratch);
  if (rc)
    return rc;
  // Every byte of the staging that is read in this call is first written in
  // this call (scans write all offsets, the gather all output entries), so
  // nothing needs clearing.
  unsigned long long* dOffsets = reinterpret_cast<unsigned long long*>(scratch);
  cudaStream_t s = ev->stream;
  const lst::EventView* v = ev->dv + first;
  LST_LAUNCH_PLAIN(lst::kOutputSizes, dim3(1, count), 1024, v);
  LST_LAUNCH_PLAIN(lst::kOutputEventOffsets, 1, 1024, v, count, dOffsets);
  LST_CUDA(cudaMemcpyAsync(out->event_tc_offsets, dOffsets, sizeof(uint64_t) * (count + 1), cudaMemcpyDeviceToHost,
                           s));
  LST_CUDA(cudaMemcpyAsync(out->event_hit_offsets, dOffsets + count + 1, sizeof(uint64_t) * (count + 1),
                           cudaMemcpyDeviceToHost, s));
  LST_CUDA(cudaStreamSynchronize(s));
  const size_t nTC = out->event_tc_offsets[count], nHits = out->event_hit_offsets[count];
  if (nTC > out->tc_capacity || nHits > out->hits_capacity)
    return setError("lst_batch_get_output_static: output capacity too small (" + std::to_string(nTC) +
                    " candidates, " + std::to_string(nHits) + " hits needed)");
  Carver need;
  need.take<unsigned int>(nHits);
  need.take<unsigned int>(nTC);
  need.take<int>(nTC);
  need.take<short>(nTC);
  if (kStaticOffsetBytes + need.off > kStaticOutputBytes)
    return setError("lst_batch_get_output_static: the output of these events needs " +
                    std::to_string(kStaticOffsetBytes + need.off) + " bytes of staging, more than the " +
                    std::to_string(kStaticOutputBytes) + "-byte static buffer (split the slot range)");
  if (nTC == 0)
    return 0;
  if (!out->hits || !out->len || !out->seedIdx || !out->type)
    return setError("lst_batch_get_output_static: null output array");
  Carver d;
  d.base = reinterpret_cast<char*>(scratch + kStaticOffsetBytes);
  unsigned int* dHits = d.take<unsigned int>(nHits);
  unsigned int* dLen = d.take<unsigned int>(nTC);
  int* dSeed = d.take<int>(nTC);
  short* dType = d.take<short>(nTC);
  LST_LAUNCH_PLAIN(lst::kOutputGather, dim3(blocksFor(lst::kMaxTrackCandidates, count), count), kThreads, v, count,
                   dOffsets, dHits, dLen, dSeed, dType);
  LST_CUDA(cudaMemcpyAsync(out->hits, dHits, nHits * sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
  LST_CUDA(cudaMemcpyAsync(out->len, dLen, nTC * sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
  LST_CUDA(cudaMemcpyAsync(out->seedIdx, dSeed, nTC * sizeof(int), cudaMemcpyDeviceToHost, s));
  LST_CUDA(cudaMemcpyAsync(out->type, dType, nTC * sizeof(short), cudaMemcpyDeviceToHost, s));
  LST_CUDA(cudaStreamSynchronize(s));
  return 0;
  LST_ABI_CATCH_INT
}

int lst_event_launches(const lst_event* ev, uint64_t* n) {
  LST_ABI_TRY
  if (!ev || !n)
    return setError("lst_event_launches: null argument");
  *n = ev->launches;
  return 0;
  LST_ABI_CATCH_INT
}

int lst_event_set_profiling(lst_event* ev, int on) {
  LST_ABI_TRY
  if (!ev)
    return setError("null event set");
  LST_CUDA(cudaStreamSynchronize(ev->stream));
  ev->profiling = on != 0;
  ev->profile.clear();
  ev->poolUsed = 0;
  return 0;
  LST_ABI_CATCH_INT
}

int lst_event_get_profile(lst_event* ev, lst_kernel_time* out, int capacity, int* n_kernels) {
  LST_ABI_TRY
  if (!ev || !n_kernels)
    return setError("lst_event_get_profile: null argument");
  LST_CUDA(cudaStreamSynchronize(ev->stream));
  std::vector<lst_kernel_time> acc;
  for (const ProfRecord& r : ev->profile) {
    float ms = 0.f;
    LST_CUDA(cudaEventElapsedTime(&ms, r.start, r.stop));
    const char* name = r.kernel;
    if (std::strncmp(name, "lst::", 5) == 0)
      name += 5;
    auto it = std::find_if(acc.begin(), acc.end(), [&](const lst_kernel_time& k) { return std::strcmp(k.name, name) == 0; });
    if (it == acc.end()) {
      lst_kernel_time k{};
      k.name = name;
      acc.push_back(k);
      it = acc.end() - 1;
    }
    it->launches += 1;
    it->total_ms += ms;
  }
  *n_kernels = static_cast<int>(acc.size());
  for (int i = 0; i < static_cast<int>(acc.size()) && i < capacity && out; ++i)
    out[i] = acc[i];
  ev->profile.clear();
  ev->poolUsed = 0;
  return 0;
  LST_ABI_CATCH_INT
}

}  // extern "C"

// ================================================================ autotuner
namespace {
  // FNV-1a over the arrays that define the geometry and the static arenas.
  template <typename T>
  void fnv(uint64_t& h, const std::vector<T>& v) {
    const unsigned char* p = reinterpret_cast<const unsigned char*>(v.data());
    for (size_t i = 0; i < v.size() * sizeof(T); ++i) {
      h ^= p[i];
      h *= 1099511628211ull;
    }
  }
  uint64_t geometryHash(const lst_es* es) {
    uint64_t h = 1469598103934665603ull;
    const lst::EsHost& g = es->host;
    fnv(h, g.detIds);
    fnv(h, g.moduleMap);
    fnv(h, g.nConnectedModules);
    fnv(h, g.connectedPixels);
    fnv(h, g.connectedPixelsIndex);
    fnv(h, g.mdCap);
    fnv(h, g.lsCap);
    fnv(h, g.t3CapIfUsed);
    fnv(h, g.t5CapIfEligible);
    return h;
  }

  void dropGraphs(lst_event* ev) {
    cudaStreamSynchronize(ev->stream);
    for (auto& g : ev->graphs)
      cudaGraphExecDestroy(g.second.exec);
    ev->graphs.clear();
  }

  // Cache key: geometry, device, batch size and this build of the kernels
  // (shapes tuned for one build need not suit another).
  std::string tuneKey(const lst_event* ev, int count) {
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, ev->device);
    char buf[512];
    std::snprintf(buf, sizeof(buf), "g%016llx-d%s-n%d-b%s_%s", static_cast<unsigned long long>(geometryHash(ev->es)),
                  prop.name, count, __DATE__, __TIME__);
    std::string key(buf);
    for (char& c : key)
      if (c == ' ' || c == '\t')
        c = '_';
    return key;
  }

  std::string shapesLine(const lst_event* ev) {
    std::string line;
    for (int k = 0; k < kTuCount; ++k)
      line += " " + std::string(kTuneSpecs[k].name) + "=" + std::to_string(ev->shape[k].warps) + "x" +
              std::to_string(ev->shape[k].perSM);
    return line;
  }

  // Parses the "name=WxP" fields of a cache line; false if malformed or incomplete.
  bool parseShapes(const std::string& rest, LaunchShape* out) {
    std::istringstream is(rest);
    std::string tok;
    int found = 0;
    while (is >> tok) {
      const size_t eq = tok.find('='), x = tok.rfind('x');
      if (eq == std::string::npos || x == std::string::npos || x < eq)
        return false;
      const std::string name = tok.substr(0, eq);
      int w = 0, p = 0;
      try {
        w = std::stoi(tok.substr(eq + 1, x - eq - 1));
        p = std::stoi(tok.substr(x + 1));
      } catch (...) {
        return false;
      }
      for (int k = 0; k < kTuCount; ++k) {
        if (name == kTuneSpecs[k].name) {
          if (w < 1 || w > kTuneSpecs[k].maxWarps || p < 1 || p > 256)
            return false;
          out[k].warps = w;
          out[k].perSM = p;
          ++found;
        }
      }
    }
    return found == kTuCount;
  }

  // Per-kernel device time (ms) of the launches profiled since the last clear.
  int collectProfile(lst_event* ev, std::map<std::string, double>& ms) {
    LST_CUDA(cudaStreamSynchronize(ev->stream));
    for (const ProfRecord& r : ev->profile) {
      float t = 0.f;
      LST_CUDA(cudaEventElapsedTime(&t, r.start, r.stop));
      const char* name = r.kernel;
      if (std::strncmp(name, "lst::", 5) == 0)
        name += 5;
      ms[name] += t;
    }
    ev->profile.clear();
    ev->poolUsed = 0;
    return 0;
  }
}  // namespace

extern "C" {

int lst_tune_kernel_count(void) {
  LST_ABI_TRY
  return kTuCount;
  LST_ABI_CATCH_INT
}

const char* lst_tune_kernel_name(int k) { return (k >= 0 && k < kTuCount) ? kTuneSpecs[k].name : nullptr; }

int lst_event_set_launch_shape(lst_event* ev, int k, int warps_per_block, int blocks_per_sm) {
  LST_ABI_TRY
  if (!ev)
    return setError("null event set");
  if (k < 0 || k >= kTuCount)
    return setError("lst_event_set_launch_shape: no tunable kernel " + std::to_string(k));
  if (warps_per_block < 1 || warps_per_block > kTuneSpecs[k].maxWarps)
    return setError(std::string("lst_event_set_launch_shape: ") + kTuneSpecs[k].name + " takes 1.." +
                    std::to_string(kTuneSpecs[k].maxWarps) + " warps per block");
  if (blocks_per_sm < 1 || blocks_per_sm > 256)
    return setError("lst_event_set_launch_shape: blocks per SM must be 1..256");
  if (ev->shape[k].warps != warps_per_block || ev->shape[k].perSM != blocks_per_sm) {
    dropGraphs(ev);
    ev->shape[k].warps = warps_per_block;
    ev->shape[k].perSM = blocks_per_sm;
  }
  return 0;
  LST_ABI_CATCH_INT
}

int lst_event_get_launch_shape(const lst_event* ev, int k, int* warps_per_block, int* blocks_per_sm) {
  LST_ABI_TRY
  if (!ev || !warps_per_block || !blocks_per_sm)
    return setError("lst_event_get_launch_shape: null argument");
  if (k < 0 || k >= kTuCount)
    return setError("lst_event_get_launch_shape: no tunable kernel " + std::to_string(k));
  *warps_per_block = ev->shape[k].warps;
  *blocks_per_sm = ev->shape[k].perSM;
  return 0;
  LST_ABI_CATCH_INT
}

uint64_t lst_es_geometry_hash(const lst_es* es) {
  try {
    return es ? geometryHash(es) : 0;
  } catch (...) {
    return 0;
  }
}

int lst_autotune_load(lst_event* ev, int count, const char* cache_path) {
  LST_ABI_TRY
  if (!ev || !cache_path)
    return setError("lst_autotune_load: null argument");
  std::ifstream in(cache_path);
  if (!in)
    return 0;
  const std::string key = tuneKey(ev, count);
  std::string line, found;
  while (std::getline(in, line))
    if (line.compare(0, key.size() + 1, key + " ") == 0)
      found = line.substr(key.size() + 1);
  if (found.empty())
    return 0;
  LaunchShape shapes[kTuCount];
  if (!parseShapes(found, shapes))
    return setError("lst_autotune_load: malformed entry for " + key + " in " + cache_path);
  for (int k = 0; k < kTuCount; ++k) {
    int rc = lst_event_set_launch_shape(ev, k, shapes[k].warps, shapes[k].perSM);
    if (rc)
      return rc;
  }
  return 1;
  LST_ABI_CATCH_INT
}

int lst_autotune(lst_event* ev, int first, int count, const char* cache_path) {
  LST_ABI_TRY
  int rc = checkSlots(ev, first, count);
  if (rc)
    return rc;
  if (count == 0)
    return 0;
  if (!ev->inboxValid || first < ev->inboxFirst || first + count > ev->inboxFirst + ev->inboxCount)
    return setError("lst_autotune: upload the calibration events into slots [first, first + count) first");
  const bool wasProfiling = ev->profiling;
  LaunchShape saved[kTuCount];
  std::copy(ev->shape, ev->shape + kTuCount, saved);
  auto restore = [&]() {
    for (int k = 0; k < kTuCount; ++k)
      lst_event_set_launch_shape(ev, k, saved[k].warps, saved[k].perSM);
    ev->profiling = wasProfiling;
    ev->profile.clear();
    ev->poolUsed = 0;
  };
  std::vector<lst_counts> refCounts(count), counts(count);
  ev->profiling = false;
  if ((rc = ingestInbox(ev, first, count)) || (rc = lst_batch_run(ev, first, count, 1, 8)) ||
      (rc = readCounts(ev, first, count, refCounts.data()))) {
    restore();
    return rc;
  }
  const int warpOpts[] = {1, 2, 4, 8};
  const int perSMOpts[] = {16, 32, 64, 128};
  struct Trial {
    int w, p;
  };
  std::vector<Trial> trials;
  for (int w : warpOpts)
    for (int p : perSMOpts)
      trials.push_back({w, p});
  std::vector<std::vector<double>> best(kTuCount, std::vector<double>(trials.size(), 1e30));
  for (int rep = 0; rep < 2; ++rep) {
    for (size_t t = 0; t < trials.size(); ++t) {
      for (int k = 0; k < kTuCount; ++k)
        lst_event_set_launch_shape(ev, k, std::min(trials[t].w, kTuneSpecs[k].maxWarps), trials[t].p);
      ev->profiling = false;
      if ((rc = ingestInbox(ev, first, count))) {
        restore();
        return rc;
      }
      if (cudaStreamSynchronize(ev->stream) != cudaSuccess) {
        restore();
        return cudaFail(cudaGetLastError(), "lst_autotune");
      }
      ev->profile.clear();
      ev->poolUsed = 0;
      ev->profiling = true;
      rc = lst_batch_run(ev, first, count, 1, 8);
      std::map<std::string, double> ms;
      if (!rc)
        rc = collectProfile(ev, ms);
      ev->profiling = false;
      if (!rc)
        rc = readCounts(ev, first, count, counts.data());
      if (rc) {
        restore();
        return rc;
      }
      if (std::memcmp(counts.data(), refCounts.data(), sizeof(lst_counts) * count) != 0) {
        restore();
        return setError("lst_autotune: the object counts changed with the launch shape (" +
                        std::to_string(trials[t].w) + " warps, " + std::to_string(trials[t].p) +
                        " blocks per SM)");
      }
      for (int k = 0; k < kTuCount; ++k) {
        if (trials[t].w > kTuneSpecs[k].maxWarps)
          continue;  // this kernel ran the shape of another trial
        auto it = ms.find(kTuneSpecs[k].name);
        if (it != ms.end())
          best[k][t] = std::min(best[k][t], it->second);
      }
    }
  }
  ev->profiling = wasProfiling;
  for (int k = 0; k < kTuCount; ++k) {
    size_t arg = 0;
    for (size_t t = 1; t < trials.size(); ++t)
      if (best[k][t] < best[k][arg])
        arg = t;
    if (best[k][arg] >= 1e30)  // never timed: keep the previous shape
      lst_event_set_launch_shape(ev, k, saved[k].warps, saved[k].perSM);
    else
      lst_event_set_launch_shape(ev, k, trials[arg].w, trials[arg].p);
  }
  if (cache_path && *cache_path) {
    const std::string key = tuneKey(ev, count);
    std::vector<std::string> lines;
    {
      std::ifstream in(cache_path);
      std::string line;
      while (std::getline(in, line))
        if (!line.empty() && line.compare(0, key.size() + 1, key + " ") != 0)
          lines.push_back(line);
    }
    lines.push_back(key + shapesLine(ev));
    const std::string tmp = std::string(cache_path) + ".tmp";
    {
      std::ofstream out(tmp, std::ios::trunc);
      if (!out)
        return setError(std::string("lst_autotune: cannot write ") + tmp);
      for (const std::string& l : lines)
        out << l << "\n";
    }
    if (std::rename(tmp.c_str(), cache_path) != 0)
      return setError(std::string("lst_autotune: cannot replace ") + cache_path);
  }
  return 0;
  LST_ABI_CATCH_INT
}

}  // extern "C"
