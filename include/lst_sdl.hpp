/* lst_sdl.hpp -- the reference's C++ surface (SDL::Event<SDL::Acc>,
 * SDL::LST<SDL::Acc>, the event-setup loaders) over the C ABI of lst_b200.h,
 * so that caller source written against the reference compiles unchanged and
 * runs on the B200 library.
 *
 * Replaces, for callers:
 *   SDL/Event.h:31-205      SDL::Event<SDL::Acc> (ctor, addHitToEvent,
 *                           addPixelSegmentToEvent, the create* stages,
 *                           pixelLineSegmentCleaning, getNumberOf*, the
 *                           get* host-buffer getters, resetEvent)
 *   SDL/LST.h:25-111        SDL::LST<SDL::Acc>::run(queue, verbose, es, ...)
 *                           and hits() / len() / seedIdx() /
 *                           trackCandidateType()
 *   SDL/LSTESData.h:79-80   SDL::loadAndFillESHost, SDL::loadAndFillESDevice
 *
 * The Alpaka types the reference's signatures name are stand-ins here:
 * SDL::QueueAcc holds a CUDA stream (as void*) and a device ordinal, SDL::Acc
 * and SDL::Dev are tags, alpaka::DevCpu a tag for the host buffers.  A
 * translation unit uses either this header or the reference's Alpaka headers.
 *
 * Errors of the C ABI become std::runtime_error with lst_last_error()'s text
 * (the reference throws on bad geometry files too).  Host buffers returned by
 * the get* getters stay valid until resetEvent() or the Event's destruction,
 * as in the reference (SDL/Event.cc:1489-1814). */
#ifndef LST_SDL_HPP
#define LST_SDL_HPP

#include <cstdint>
#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "lst_b200.h"

namespace alpaka {
  struct DevCpu;  // tag: the host copies the getters return
}

namespace SDL {

  struct AccTag {};
  struct DevTag {};
  using Acc = AccTag;
  using Dev = DevTag;

  // The queue the reference passes around: here a CUDA stream (cudaStream_t
  // as void*, nullptr = the library's own stream) on a device.
  struct QueueAcc {
    void* stream = nullptr;
    int device = 0;
  };

  inline void lstCheck(int rc) {
    if (rc < 0)
      throw std::runtime_error(lst_last_error());
  }

  // ------------------------------------------------------- event setup
  template <typename>
  struct LSTESHostData;
  template <>
  struct LSTESHostData<Dev> {
    std::string geometryDir;   // <LST_BASE>/data/OT800_IT615_pt0.8
    std::string t5dnnWeights;  // <LST_BASE>/data/t5dnn_reference.bin
  };

  template <typename>
  struct LSTESDeviceData;
  template <>
  struct LSTESDeviceData<Dev> {
    uint16_t nModules = 0;
    uint16_t nLowerModules = 0;
    unsigned int nPixels = 0;
    std::shared_ptr<lst_es> es;  // read-only, shared by every Event and LST
  };

  // SDL/LSTESData.cc:14-75 reads $LST_BASE/data/OT800_IT615_pt0.8; the
  // classifier weights ship beside it as a file.
  inline std::unique_ptr<LSTESHostData<Dev>> loadAndFillESHost() {
    const char* base = std::getenv("LST_BASE");
    if (!base)
      throw std::runtime_error("LST_BASE is not set");
    auto h = std::make_unique<LSTESHostData<Dev>>();
    h->geometryDir = std::string(base) + "/data/OT800_IT615_pt0.8";
    h->t5dnnWeights = std::string(base) + "/data/t5dnn_reference.bin";
    return h;
  }

  inline std::unique_ptr<LSTESDeviceData<Dev>> loadAndFillESDevice(QueueAcc& queue,
                                                                    const LSTESHostData<Dev>* hostData) {
    lst_es* es = nullptr;
    lstCheck(lst_es_load(hostData->geometryDir.c_str(), hostData->t5dnnWeights.c_str(), queue.device, &es));
    auto d = std::make_unique<LSTESDeviceData<Dev>>();
    d->es = std::shared_ptr<lst_es>(es, [](lst_es* p) { lst_es_free(p); });
    lst_es_info info;
    lstCheck(lst_es_get_info(es, &info));
    d->nModules = static_cast<uint16_t>(info.nModules);
    d->nLowerModules = static_cast<uint16_t>(info.nLowerModules);
    d->nPixels = info.nConnectedPixels;
    return d;
  }

  // ------------------------------------------------------ host buffers
  struct LSTuint4 {
    unsigned int x, y, z, w;
  };

  // SDL::hits (field names and types as in the reference's store)
  struct hits {
    float* xs = nullptr;
    float* ys = nullptr;
    float* zs = nullptr;
    uint16_t* moduleIndices = nullptr;
    unsigned int* idxs = nullptr;
    unsigned int* detid = nullptr;
    float* rts = nullptr;
    float* phis = nullptr;
    float* etas = nullptr;
    float* highEdgeXs = nullptr;
    float* highEdgeYs = nullptr;
    float* lowEdgeXs = nullptr;
    float* lowEdgeYs = nullptr;
    int* hitRanges = nullptr;
    int* hitRangesLower = nullptr;
    int* hitRangesUpper = nullptr;
    int8_t* hitRangesnLower = nullptr;
    int8_t* hitRangesnUpper = nullptr;
  };

  // SDL::miniDoublets (field names and types as in the reference's store)
  struct miniDoublets {
    unsigned int* anchorHitIndices = nullptr;
    unsigned int* outerHitIndices = nullptr;
    uint16_t* moduleIndices = nullptr;
    unsigned int* nMDs = nullptr;
    unsigned int* totOccupancyMDs = nullptr;
    float* dphichanges = nullptr;
    float* dzs = nullptr;
    float* dphis = nullptr;
    float* shiftedXs = nullptr;
    float* shiftedYs = nullptr;
    float* shiftedZs = nullptr;
    float* noShiftedDzs = nullptr;
    float* noShiftedDphis = nullptr;
    float* noShiftedDphiChanges = nullptr;
    float* anchorX = nullptr;
    float* anchorY = nullptr;
    float* anchorZ = nullptr;
    float* anchorRt = nullptr;
    float* anchorPhi = nullptr;
    float* anchorEta = nullptr;
    float* anchorHighEdgeX = nullptr;
    float* anchorHighEdgeY = nullptr;
    float* anchorLowEdgeX = nullptr;
    float* anchorLowEdgeY = nullptr;
    float* anchorLowEdgePhi = nullptr;
    float* anchorHighEdgePhi = nullptr;
    float* outerX = nullptr;
    float* outerY = nullptr;
    float* outerZ = nullptr;
    float* outerRt = nullptr;
    float* outerPhi = nullptr;
    float* outerEta = nullptr;
    float* outerHighEdgeX = nullptr;
    float* outerHighEdgeY = nullptr;
    float* outerLowEdgeX = nullptr;
    float* outerLowEdgeY = nullptr;
  };

  // SDL::segments (field names and types as in the reference's store)
  struct segments {
    float* dPhis = nullptr;
    float* dPhiMins = nullptr;
    float* dPhiMaxs = nullptr;
    float* dPhiChanges = nullptr;
    float* dPhiChangeMins = nullptr;
    float* dPhiChangeMaxs = nullptr;
    uint16_t* innerLowerModuleIndices = nullptr;
    uint16_t* outerLowerModuleIndices = nullptr;
    unsigned int* mdIndices = nullptr;
    unsigned int* innerMiniDoubletAnchorHitIndices = nullptr;
    unsigned int* outerMiniDoubletAnchorHitIndices = nullptr;
    unsigned int* nSegments = nullptr;
    unsigned int* totOccupancySegments = nullptr;
    unsigned int* seedIdx = nullptr;
    int* charge = nullptr;
    int* superbin = nullptr;
    LSTuint4* pLSHitsIdxs = nullptr;
    int8_t* pixelType = nullptr;
    int8_t* isQuad = nullptr;
    int8_t* isDup = nullptr;
    uint8_t* partOfPT5 = nullptr;
    float* ptIn = nullptr;
    float* ptErr = nullptr;
    float* px = nullptr;
    float* py = nullptr;
    float* pz = nullptr;
    float* etaErr = nullptr;
    float* eta = nullptr;
    float* phi = nullptr;
    float* score = nullptr;
    float* circleCenterX = nullptr;
    float* circleCenterY = nullptr;
    float* circleRadius = nullptr;
  };

  // SDL::triplets (field names and types as in the reference's store)
  struct triplets {
    unsigned int* segmentIndices = nullptr;
    uint16_t* lowerModuleIndices = nullptr;
    unsigned int* nTriplets = nullptr;
    unsigned int* totOccupancyTriplets = nullptr;
    uint8_t* logicalLayers = nullptr;
    unsigned int* hitIndices = nullptr;
    float* betaIn = nullptr;
    float* circleRadius = nullptr;
    float* circleCenterX = nullptr;
    float* circleCenterY = nullptr;
    uint8_t* partOfPT5 = nullptr;
    uint8_t* partOfT5 = nullptr;
    uint8_t* partOfPT3 = nullptr;
  };

  // SDL::quintuplets (field names and types as in the reference's store)
  struct quintuplets {
    unsigned int* tripletIndices = nullptr;
    uint16_t* lowerModuleIndices = nullptr;
    unsigned int* nQuintuplets = nullptr;
    unsigned int* totOccupancyQuintuplets = nullptr;
    float* innerRadius = nullptr;
    float* bridgeRadius = nullptr;
    float* outerRadius = nullptr;
    float* pt = nullptr;
    float* eta = nullptr;
    float* phi = nullptr;
    float* score_rphisum = nullptr;
    uint8_t* layer = nullptr;
    int8_t* isDup = nullptr;
    uint8_t* TightCutFlag = nullptr;
    uint8_t* partOfPT5 = nullptr;
    float* regressionRadius = nullptr;
    float* regressionG = nullptr;
    float* regressionF = nullptr;
    uint8_t* logicalLayers = nullptr;
    unsigned int* hitIndices = nullptr;
    float* rzChiSquared = nullptr;
    float* chiSquared = nullptr;
    float* nonAnchorChiSquared = nullptr;
  };

  // SDL::pixelTriplets (field names and types as in the reference's store)
  struct pixelTriplets {
    unsigned int* pixelSegmentIndices = nullptr;
    unsigned int* tripletIndices = nullptr;
    unsigned int* nPixelTriplets = nullptr;
    unsigned int* totOccupancyPixelTriplets = nullptr;
    float* pixelRadius = nullptr;
    float* tripletRadius = nullptr;
    float* pt = nullptr;
    float* eta = nullptr;
    float* phi = nullptr;
    float* eta_pix = nullptr;
    float* phi_pix = nullptr;
    float* score = nullptr;
    uint8_t* isDup = nullptr;
    uint8_t* partOfPT5 = nullptr;
    uint8_t* logicalLayers = nullptr;
    unsigned int* hitIndices = nullptr;
    uint16_t* lowerModuleIndices = nullptr;
    float* centerX = nullptr;
    float* centerY = nullptr;
    float* pixelRadiusError = nullptr;
    float* rPhiChiSquared = nullptr;
    float* rPhiChiSquaredInwards = nullptr;
    float* rzChiSquared = nullptr;
  };

  // SDL::pixelQuintuplets (field names and types as in the reference's store)
  struct pixelQuintuplets {
    unsigned int* pixelIndices = nullptr;
    unsigned int* T5Indices = nullptr;
    unsigned int* nPixelQuintuplets = nullptr;
    unsigned int* totOccupancyPixelQuintuplets = nullptr;
    uint8_t* isDup = nullptr;
    float* score = nullptr;
    float* eta = nullptr;
    float* phi = nullptr;
    uint8_t* logicalLayers = nullptr;
    unsigned int* hitIndices = nullptr;
    uint16_t* lowerModuleIndices = nullptr;
    float* pixelRadius = nullptr;
    float* quintupletRadius = nullptr;
    float* centerX = nullptr;
    float* centerY = nullptr;
    float* rzChiSquared = nullptr;
    float* rPhiChiSquared = nullptr;
    float* rPhiChiSquaredInwards = nullptr;
  };

  // SDL::trackCandidates (field names and types as in the reference's store)
  struct trackCandidates {
    short* trackCandidateType = nullptr;
    unsigned int* directObjectIndices = nullptr;
    unsigned int* objectIndices = nullptr;
    unsigned int* nTrackCandidates = nullptr;
    unsigned int* nTrackCandidatespT3 = nullptr;
    unsigned int* nTrackCandidatespT5 = nullptr;
    unsigned int* nTrackCandidatespLS = nullptr;
    unsigned int* nTrackCandidatesT5 = nullptr;
    uint8_t* logicalLayers = nullptr;
    unsigned int* hitIndices = nullptr;
    int* pixelSeedIndex = nullptr;
    uint16_t* lowerModuleIndices = nullptr;
    float* centerX = nullptr;
    float* centerY = nullptr;
    float* radius = nullptr;
  };

  // SDL::objectRanges (field names and types as in the reference's store)
  struct objectRanges {
    int* mdRanges = nullptr;
    int* segmentRanges = nullptr;
    int* tripletRanges = nullptr;
    int* quintupletRanges = nullptr;
    uint16_t* nEligibleT5Modules = nullptr;
    uint16_t* indicesOfEligibleT5Modules = nullptr;
    int* quintupletModuleIndices = nullptr;
    int* quintupletModuleOccupancy = nullptr;
    int* miniDoubletModuleIndices = nullptr;
    int* miniDoubletModuleOccupancy = nullptr;
    int* segmentModuleIndices = nullptr;
    int* segmentModuleOccupancy = nullptr;
    int* tripletModuleIndices = nullptr;
    int* tripletModuleOccupancy = nullptr;
    unsigned int* device_nTotalMDs = nullptr;
    unsigned int* device_nTotalSegs = nullptr;
    unsigned int* device_nTotalTrips = nullptr;
    unsigned int* device_nTotalQuints = nullptr;
  };

  template <typename TDev>
  struct hitsBuffer : hits {};
  template <typename TDev>
  struct miniDoubletsBuffer : miniDoublets {};
  template <typename TDev>
  struct segmentsBuffer : segments {};
  template <typename TDev>
  struct tripletsBuffer : triplets {};
  template <typename TDev>
  struct quintupletsBuffer : quintuplets {};
  template <typename TDev>
  struct pixelTripletsBuffer : pixelTriplets {};
  template <typename TDev>
  struct pixelQuintupletsBuffer : pixelQuintuplets {};
  template <typename TDev>
  struct trackCandidatesBuffer : trackCandidates {};
  template <typename TDev>
  struct objectRangesBuffer : objectRanges {};

#define LST_SDL_STORE_FIELDS(X) \
  X(hits, "hits.", xs) \
  X(hits, "hits.", ys) \
  X(hits, "hits.", zs) \
  X(hits, "hits.", moduleIndices) \
  X(hits, "hits.", idxs) \
  X(hits, "hits.", detid) \
  X(hits, "hits.", rts) \
  X(hits, "hits.", phis) \
  X(hits, "hits.", etas) \
  X(hits, "hits.", highEdgeXs) \
  X(hits, "hits.", highEdgeYs) \
  X(hits, "hits.", lowEdgeXs) \
  X(hits, "hits.", lowEdgeYs) \
  X(hits, "hits.", hitRanges) \
  X(hits, "hits.", hitRangesLower) \
  X(hits, "hits.", hitRangesUpper) \
  X(hits, "hits.", hitRangesnLower) \
  X(hits, "hits.", hitRangesnUpper) \
  X(miniDoublets, "md.", anchorHitIndices) \
  X(miniDoublets, "md.", outerHitIndices) \
  X(miniDoublets, "md.", moduleIndices) \
  X(miniDoublets, "md.", nMDs) \
  X(miniDoublets, "md.", totOccupancyMDs) \
  X(miniDoublets, "md.", dphichanges) \
  X(miniDoublets, "md.", dzs) \
  X(miniDoublets, "md.", dphis) \
  X(miniDoublets, "md.", shiftedXs) \
  X(miniDoublets, "md.", shiftedYs) \
  X(miniDoublets, "md.", shiftedZs) \
  X(miniDoublets, "md.", noShiftedDzs) \
  X(miniDoublets, "md.", noShiftedDphis) \
  X(miniDoublets, "md.", noShiftedDphiChanges) \
  X(miniDoublets, "md.", anchorX) \
  X(miniDoublets, "md.", anchorY) \
  X(miniDoublets, "md.", anchorZ) \
  X(miniDoublets, "md.", anchorRt) \
  X(miniDoublets, "md.", anchorPhi) \
  X(miniDoublets, "md.", anchorEta) \
  X(miniDoublets, "md.", anchorHighEdgeX) \
  X(miniDoublets, "md.", anchorHighEdgeY) \
  X(miniDoublets, "md.", anchorLowEdgeX) \
  X(miniDoublets, "md.", anchorLowEdgeY) \
  X(miniDoublets, "md.", anchorLowEdgePhi) \
  X(miniDoublets, "md.", anchorHighEdgePhi) \
  X(miniDoublets, "md.", outerX) \
  X(miniDoublets, "md.", outerY) \
  X(miniDoublets, "md.", outerZ) \
  X(miniDoublets, "md.", outerRt) \
  X(miniDoublets, "md.", outerPhi) \
  X(miniDoublets, "md.", outerEta) \
  X(miniDoublets, "md.", outerHighEdgeX) \
  X(miniDoublets, "md.", outerHighEdgeY) \
  X(miniDoublets, "md.", outerLowEdgeX) \
  X(miniDoublets, "md.", outerLowEdgeY) \
  X(segments, "ls.", dPhis) \
  X(segments, "ls.", dPhiMins) \
  X(segments, "ls.", dPhiMaxs) \
  X(segments, "ls.", dPhiChanges) \
  X(segments, "ls.", dPhiChangeMins) \
  X(segments, "ls.", dPhiChangeMaxs) \
  X(segments, "ls.", innerLowerModuleIndices) \
  X(segments, "ls.", outerLowerModuleIndices) \
  X(segments, "ls.", mdIndices) \
  X(segments, "ls.", innerMiniDoubletAnchorHitIndices) \
  X(segments, "ls.", outerMiniDoubletAnchorHitIndices) \
  X(segments, "ls.", nSegments) \
  X(segments, "ls.", totOccupancySegments) \
  X(segments, "ls.", seedIdx) \
  X(segments, "ls.", charge) \
  X(segments, "ls.", superbin) \
  X(segments, "ls.", pLSHitsIdxs) \
  X(segments, "ls.", pixelType) \
  X(segments, "ls.", isQuad) \
  X(segments, "ls.", isDup) \
  X(segments, "ls.", partOfPT5) \
  X(segments, "ls.", ptIn) \
  X(segments, "ls.", ptErr) \
  X(segments, "ls.", px) \
  X(segments, "ls.", py) \
  X(segments, "ls.", pz) \
  X(segments, "ls.", etaErr) \
  X(segments, "ls.", eta) \
  X(segments, "ls.", phi) \
  X(segments, "ls.", score) \
  X(segments, "ls.", circleCenterX) \
  X(segments, "ls.", circleCenterY) \
  X(segments, "ls.", circleRadius) \
  X(triplets, "t3.", segmentIndices) \
  X(triplets, "t3.", lowerModuleIndices) \
  X(triplets, "t3.", nTriplets) \
  X(triplets, "t3.", totOccupancyTriplets) \
  X(triplets, "t3.", logicalLayers) \
  X(triplets, "t3.", hitIndices) \
  X(triplets, "t3.", betaIn) \
  X(triplets, "t3.", circleRadius) \
  X(triplets, "t3.", circleCenterX) \
  X(triplets, "t3.", circleCenterY) \
  X(triplets, "t3.", partOfPT5) \
  X(triplets, "t3.", partOfT5) \
  X(triplets, "t3.", partOfPT3) \
  X(quintuplets, "t5.", tripletIndices) \
  X(quintuplets, "t5.", lowerModuleIndices) \
  X(quintuplets, "t5.", nQuintuplets) \
  X(quintuplets, "t5.", totOccupancyQuintuplets) \
  X(quintuplets, "t5.", innerRadius) \
  X(quintuplets, "t5.", bridgeRadius) \
  X(quintuplets, "t5.", outerRadius) \
  X(quintuplets, "t5.", pt) \
  X(quintuplets, "t5.", eta) \
  X(quintuplets, "t5.", phi) \
  X(quintuplets, "t5.", score_rphisum) \
  X(quintuplets, "t5.", layer) \
  X(quintuplets, "t5.", isDup) \
  X(quintuplets, "t5.", TightCutFlag) \
  X(quintuplets, "t5.", partOfPT5) \
  X(quintuplets, "t5.", regressionRadius) \
  X(quintuplets, "t5.", regressionG) \
  X(quintuplets, "t5.", regressionF) \
  X(quintuplets, "t5.", logicalLayers) \
  X(quintuplets, "t5.", hitIndices) \
  X(quintuplets, "t5.", rzChiSquared) \
  X(quintuplets, "t5.", chiSquared) \
  X(quintuplets, "t5.", nonAnchorChiSquared) \
  X(pixelTriplets, "pt3.", pixelSegmentIndices) \
  X(pixelTriplets, "pt3.", tripletIndices) \
  X(pixelTriplets, "pt3.", nPixelTriplets) \
  X(pixelTriplets, "pt3.", totOccupancyPixelTriplets) \
  X(pixelTriplets, "pt3.", pixelRadius) \
  X(pixelTriplets, "pt3.", tripletRadius) \
  X(pixelTriplets, "pt3.", pt) \
  X(pixelTriplets, "pt3.", eta) \
  X(pixelTriplets, "pt3.", phi) \
  X(pixelTriplets, "pt3.", eta_pix) \
  X(pixelTriplets, "pt3.", phi_pix) \
  X(pixelTriplets, "pt3.", score) \
  X(pixelTriplets, "pt3.", isDup) \
  X(pixelTriplets, "pt3.", partOfPT5) \
  X(pixelTriplets, "pt3.", logicalLayers) \
  X(pixelTriplets, "pt3.", hitIndices) \
  X(pixelTriplets, "pt3.", lowerModuleIndices) \
  X(pixelTriplets, "pt3.", centerX) \
  X(pixelTriplets, "pt3.", centerY) \
  X(pixelTriplets, "pt3.", pixelRadiusError) \
  X(pixelTriplets, "pt3.", rPhiChiSquared) \
  X(pixelTriplets, "pt3.", rPhiChiSquaredInwards) \
  X(pixelTriplets, "pt3.", rzChiSquared) \
  X(pixelQuintuplets, "pt5.", pixelIndices) \
  X(pixelQuintuplets, "pt5.", T5Indices) \
  X(pixelQuintuplets, "pt5.", nPixelQuintuplets) \
  X(pixelQuintuplets, "pt5.", totOccupancyPixelQuintuplets) \
  X(pixelQuintuplets, "pt5.", isDup) \
  X(pixelQuintuplets, "pt5.", score) \
  X(pixelQuintuplets, "pt5.", eta) \
  X(pixelQuintuplets, "pt5.", phi) \
  X(pixelQuintuplets, "pt5.", logicalLayers) \
  X(pixelQuintuplets, "pt5.", hitIndices) \
  X(pixelQuintuplets, "pt5.", lowerModuleIndices) \
  X(pixelQuintuplets, "pt5.", pixelRadius) \
  X(pixelQuintuplets, "pt5.", quintupletRadius) \
  X(pixelQuintuplets, "pt5.", centerX) \
  X(pixelQuintuplets, "pt5.", centerY) \
  X(pixelQuintuplets, "pt5.", rzChiSquared) \
  X(pixelQuintuplets, "pt5.", rPhiChiSquared) \
  X(pixelQuintuplets, "pt5.", rPhiChiSquaredInwards) \
  X(trackCandidates, "tc.", trackCandidateType) \
  X(trackCandidates, "tc.", directObjectIndices) \
  X(trackCandidates, "tc.", objectIndices) \
  X(trackCandidates, "tc.", nTrackCandidates) \
  X(trackCandidates, "tc.", nTrackCandidatespT3) \
  X(trackCandidates, "tc.", nTrackCandidatespT5) \
  X(trackCandidates, "tc.", nTrackCandidatespLS) \
  X(trackCandidates, "tc.", nTrackCandidatesT5) \
  X(trackCandidates, "tc.", logicalLayers) \
  X(trackCandidates, "tc.", hitIndices) \
  X(trackCandidates, "tc.", pixelSeedIndex) \
  X(trackCandidates, "tc.", lowerModuleIndices) \
  X(trackCandidates, "tc.", centerX) \
  X(trackCandidates, "tc.", centerY) \
  X(trackCandidates, "tc.", radius) \
  X(objectRanges, "ranges.", mdRanges) \
  X(objectRanges, "ranges.", segmentRanges) \
  X(objectRanges, "ranges.", tripletRanges) \
  X(objectRanges, "ranges.", quintupletRanges) \
  X(objectRanges, "ranges.", nEligibleT5Modules) \
  X(objectRanges, "ranges.", indicesOfEligibleT5Modules) \
  X(objectRanges, "ranges.", quintupletModuleIndices) \
  X(objectRanges, "ranges.", quintupletModuleOccupancy) \
  X(objectRanges, "ranges.", miniDoubletModuleIndices) \
  X(objectRanges, "ranges.", miniDoubletModuleOccupancy) \
  X(objectRanges, "ranges.", segmentModuleIndices) \
  X(objectRanges, "ranges.", segmentModuleOccupancy) \
  X(objectRanges, "ranges.", tripletModuleIndices) \
  X(objectRanges, "ranges.", tripletModuleOccupancy) \
  X(objectRanges, "ranges.", device_nTotalMDs) \
  X(objectRanges, "ranges.", device_nTotalSegs) \
  X(objectRanges, "ranges.", device_nTotalTrips) \
  X(objectRanges, "ranges.", device_nTotalQuints)

  // ------------------------------------------------------------- Event
  template <typename>
  class Event;

  template <>
  class Event<Acc> {
  public:
    // SDL/Event.h:100-111.  maxHits bounds the hits (outer-tracker hits plus
    // pixel pseudo-hits) one event may add; the device arenas are allocated
    // once here and reused by every event (the reference allocates per event).
    template <typename TQueue>
    Event(bool verbose, TQueue const& q, const LSTESDeviceData<Dev>* deviceESData, uint32_t maxHits = 1u << 19)
        : verbose_(verbose), es_(deviceESData->es) {
      lstCheck(lst_event_create(es_.get(), 1, maxHits, q.stream, &ev_));
    }
    ~Event() { lst_event_destroy(ev_); }
    Event(const Event&) = delete;
    Event& operator=(const Event&) = delete;

    void resetEvent() {
      lstCheck(lst_event_reset(ev_, 0));
      dropHostCopies();
    }

    void addHitToEvent(std::vector<float> x,
                       std::vector<float> y,
                       std::vector<float> z,
                       std::vector<unsigned int> detId,
                       std::vector<unsigned int> idxInNtuple) {
      dropHostCopies();
      lstCheck(lst_event_add_hits(ev_, 0, static_cast<uint32_t>(x.size()), x.data(), y.data(), z.data(), detId.data(),
                                  idxInNtuple.data()));
    }

    void addPixelSegmentToEvent(std::vector<unsigned int> hitIndices0,
                                std::vector<unsigned int> hitIndices1,
                                std::vector<unsigned int> hitIndices2,
                                std::vector<unsigned int> hitIndices3,
                                std::vector<float> dPhiChange,
                                std::vector<float> ptIn,
                                std::vector<float> ptErr,
                                std::vector<float> px,
                                std::vector<float> py,
                                std::vector<float> pz,
                                std::vector<float> eta,
                                std::vector<float> etaErr,
                                std::vector<float> phi,
                                std::vector<int> charge,
                                std::vector<unsigned int> seedIdx,
                                std::vector<int> superbin,
                                std::vector<int8_t> pixelType,
                                std::vector<char> isQuad) {
      dropHostCopies();
      lstCheck(lst_event_add_pixel_segments(ev_, 0, static_cast<uint32_t>(ptIn.size()), hitIndices0.data(),
                                            hitIndices1.data(), hitIndices2.data(), hitIndices3.data(),
                                            dPhiChange.data(), ptIn.data(), ptErr.data(), px.data(), py.data(),
                                            pz.data(), eta.data(), etaErr.data(), phi.data(), charge.data(),
                                            seedIdx.data(), superbin.data(), pixelType.data(),
                                            reinterpret_cast<const int8_t*>(isQuad.data())));
    }

    void createMiniDoublets() { stage(lst_event_create_mini_doublets(ev_, 0)); }
    void createSegmentsWithModuleMap() { stage(lst_event_create_segments(ev_, 0)); }
    void createTriplets() { stage(lst_event_create_triplets(ev_, 0)); }
    void createQuintuplets() { stage(lst_event_create_quintuplets(ev_, 0)); }
    void pixelLineSegmentCleaning() { stage(lst_event_pixel_line_segment_cleaning(ev_, 0)); }
    void createPixelQuintuplets() { stage(lst_event_create_pixel_quintuplets(ev_, 0)); }
    void createPixelTriplets() { stage(lst_event_create_pixel_triplets(ev_, 0)); }
    void createTrackCandidates() { stage(lst_event_create_track_candidates(ev_, 0)); }

    // SDL/Event.cc:1263-1487
    unsigned int getNumberOfHits() { return counts().nHits; }
    unsigned int getNumberOfMiniDoublets() { return counts().nMiniDoublets; }
    unsigned int getNumberOfMiniDoubletsByLayerBarrel(unsigned int layer) { return counts().mdBarrel[layer]; }
    unsigned int getNumberOfMiniDoubletsByLayerEndcap(unsigned int layer) { return counts().mdEndcap[layer]; }
    unsigned int getNumberOfSegments() { return counts().nSegments; }
    unsigned int getNumberOfSegmentsByLayerBarrel(unsigned int layer) { return counts().lsBarrel[layer]; }
    unsigned int getNumberOfSegmentsByLayerEndcap(unsigned int layer) { return counts().lsEndcap[layer]; }
    unsigned int getNumberOfTriplets() { return counts().nTriplets; }
    unsigned int getNumberOfTripletsByLayerBarrel(unsigned int layer) { return counts().t3Barrel[layer]; }
    unsigned int getNumberOfTripletsByLayerEndcap(unsigned int layer) { return counts().t3Endcap[layer]; }
    unsigned int getNumberOfQuintuplets() { return counts().nQuintuplets; }
    unsigned int getNumberOfQuintupletsByLayerBarrel(unsigned int layer) { return counts().t5Barrel[layer]; }
    unsigned int getNumberOfQuintupletsByLayerEndcap(unsigned int layer) { return counts().t5Endcap[layer]; }
    int getNumberOfPixelTriplets() { return static_cast<int>(counts().nPixelTriplets); }
    int getNumberOfPixelQuintuplets() { return static_cast<int>(counts().nPixelQuintuplets); }
    int getNumberOfTrackCandidates() { return static_cast<int>(counts().nTrackCandidates); }
    int getNumberOfPT5TrackCandidates() { return static_cast<int>(counts().nTrackCandidatesPT5); }
    int getNumberOfPT3TrackCandidates() { return static_cast<int>(counts().nTrackCandidatesPT3); }
    int getNumberOfT5TrackCandidates() { return static_cast<int>(counts().nTrackCandidatesT5); }
    int getNumberOfPLSTrackCandidates() { return static_cast<int>(counts().nTrackCandidatesPLS); }
    int getNumberOfPixelTrackCandidates() {
      const lst_counts c = counts();
      return static_cast<int>(c.nTrackCandidates - c.nTrackCandidatesT5);
    }

    // SDL/Event.cc:1489-1814: host copies of the stores, kept until reset.
    hitsBuffer<alpaka::DevCpu>* getHits() { return fill(hits_); }
    hitsBuffer<alpaka::DevCpu>* getHitsInCMSSW() { return fill(hits_); }
    objectRangesBuffer<alpaka::DevCpu>* getRanges() { return fill(ranges_); }
    miniDoubletsBuffer<alpaka::DevCpu>* getMiniDoublets() { return fill(mds_); }
    segmentsBuffer<alpaka::DevCpu>* getSegments() { return fill(segments_); }
    tripletsBuffer<alpaka::DevCpu>* getTriplets() { return fill(triplets_); }
    quintupletsBuffer<alpaka::DevCpu>* getQuintuplets() { return fill(quintuplets_); }
    pixelTripletsBuffer<alpaka::DevCpu>* getPixelTriplets() { return fill(pixelTriplets_); }
    pixelQuintupletsBuffer<alpaka::DevCpu>* getPixelQuintuplets() { return fill(pixelQuintuplets_); }
    trackCandidatesBuffer<alpaka::DevCpu>* getTrackCandidates() { return fill(trackCandidates_); }
    trackCandidatesBuffer<alpaka::DevCpu>* getTrackCandidatesInCMSSW() { return fill(trackCandidates_); }

    // The underlying C ABI handle (slot 0), for the batched entry points.
    lst_event* handle() { return ev_; }

  private:
    template <typename B>
    struct Cached {
      bool valid = false;
      B buf;
    };

    void stage(int rc) {
      lstCheck(rc);
      dropHostCopies();
    }

    lst_counts counts() {
      lst_counts c;
      lstCheck(lst_event_get_counts(ev_, 0, &c));
      return c;
    }

    // Copies one field into host memory owned by the Event; returns its data.
    template <typename T>
    T* field(const char* name) {
      size_t n = 0, sz = 0;
      lstCheck(lst_event_get_field(ev_, 0, name, nullptr, 0, &n, &sz));
      std::vector<unsigned char>& v = host_[name];
      v.resize(n * sz);
      if (n)
        lstCheck(lst_event_get_field(ev_, 0, name, v.data(), n, &n, &sz));
      return reinterpret_cast<T*>(v.data());
    }

    template <typename B>
    B* fill(Cached<B>& c) {
      if (!c.valid) {
#define LST_SDL_FILL(STRUCT, PREFIX, F)                                                   \
  if constexpr (std::is_base_of_v<STRUCT, B>)                                             \
    c.buf.F = field<std::remove_pointer_t<decltype(c.buf.F)>>(PREFIX #F);
        LST_SDL_STORE_FIELDS(LST_SDL_FILL)
#undef LST_SDL_FILL
        c.valid = true;
      }
      return &c.buf;
    }

    void dropHostCopies() {
      hits_.valid = ranges_.valid = mds_.valid = segments_.valid = triplets_.valid = quintuplets_.valid = false;
      pixelTriplets_.valid = pixelQuintuplets_.valid = trackCandidates_.valid = false;
      host_.clear();
    }

    bool verbose_;
    std::shared_ptr<lst_es> es_;
    lst_event* ev_ = nullptr;
    std::map<std::string, std::vector<unsigned char>> host_;
    Cached<hitsBuffer<alpaka::DevCpu>> hits_;
    Cached<objectRangesBuffer<alpaka::DevCpu>> ranges_;
    Cached<miniDoubletsBuffer<alpaka::DevCpu>> mds_;
    Cached<segmentsBuffer<alpaka::DevCpu>> segments_;
    Cached<tripletsBuffer<alpaka::DevCpu>> triplets_;
    Cached<quintupletsBuffer<alpaka::DevCpu>> quintuplets_;
    Cached<pixelTripletsBuffer<alpaka::DevCpu>> pixelTriplets_;
    Cached<pixelQuintupletsBuffer<alpaka::DevCpu>> pixelQuintuplets_;
    Cached<trackCandidatesBuffer<alpaka::DevCpu>> trackCandidates_;
  };

  // --------------------------------------------------------------- LST
  template <typename>
  class LST;

  template <>
  class LST<Acc> {
  public:
    LST() = default;
    ~LST() {
      if (ev_)
        lst_event_destroy(ev_);
    }
    LST(const LST&) = delete;
    LST& operator=(const LST&) = delete;

    // SDL/LST.h:29-50 (SDL/LST.cc:12-161): seed conversion, the eight stages
    // and getOutput, on the device.  The event set is created on the first
    // call (on that call's queue and event setup) and reused.
    void run(QueueAcc& queue,
             bool verbose,
             const LSTESDeviceData<Dev>* deviceESData,
             const std::vector<float> see_px,
             const std::vector<float> see_py,
             const std::vector<float> see_pz,
             const std::vector<float> see_dxy,
             const std::vector<float> see_dz,
             const std::vector<float> see_ptErr,
             const std::vector<float> see_etaErr,
             const std::vector<float> see_stateTrajGlbX,
             const std::vector<float> see_stateTrajGlbY,
             const std::vector<float> see_stateTrajGlbZ,
             const std::vector<float> see_stateTrajGlbPx,
             const std::vector<float> see_stateTrajGlbPy,
             const std::vector<float> see_stateTrajGlbPz,
             const std::vector<int> see_q,
             const std::vector<std::vector<int>> see_hitIdx,
             const std::vector<unsigned int> ph2_detId,
             const std::vector<float> ph2_x,
             const std::vector<float> ph2_y,
             const std::vector<float> ph2_z) {
      (void)verbose;
      if (!ev_ || es_ != deviceESData->es.get()) {
        if (ev_)
          lst_event_destroy(ev_);
        ev_ = nullptr;
        es_ = deviceESData->es.get();
        esOwner_ = deviceESData->es;
        lstCheck(lst_event_create(es_, 1, 1u << 19, queue.stream, &ev_));
      }
      std::vector<uint32_t> offsets(1, 0);
      std::vector<int32_t> idx;
      for (const auto& h : see_hitIdx) {
        idx.insert(idx.end(), h.begin(), h.end());
        offsets.push_back(static_cast<uint32_t>(idx.size()));
      }
      lst_seed_input in{};
      in.n_seeds = static_cast<uint32_t>(see_px.size());
      in.see_px = see_px.data();
      in.see_py = see_py.data();
      in.see_pz = see_pz.data();
      in.see_dxy = see_dxy.data();
      in.see_dz = see_dz.data();
      in.see_ptErr = see_ptErr.data();
      in.see_etaErr = see_etaErr.data();
      in.see_stateTrajGlbX = see_stateTrajGlbX.data();
      in.see_stateTrajGlbY = see_stateTrajGlbY.data();
      in.see_stateTrajGlbZ = see_stateTrajGlbZ.data();
      in.see_stateTrajGlbPx = see_stateTrajGlbPx.data();
      in.see_stateTrajGlbPy = see_stateTrajGlbPy.data();
      in.see_stateTrajGlbPz = see_stateTrajGlbPz.data();
      in.see_q = see_q.data();
      in.see_hitIdx_offsets = offsets.data();
      in.see_hitIdx = idx.data();
      in.n_ph2 = static_cast<uint32_t>(ph2_x.size());
      in.ph2_detId = ph2_detId.data();
      in.ph2_x = ph2_x.data();
      in.ph2_y = ph2_y.data();
      in.ph2_z = ph2_z.data();
      lstCheck(lst_run(ev_, 0, &in, nullptr));
      // LST::getOutput (SDL/LST.cc:367-427), sized from the first answer
      size_t cap = 4096;
      uint64_t tco[2] = {0, 0}, hco[2] = {0, 0};
      for (;;) {
        flat_.resize(14 * cap);
        len_.resize(cap);
        seed_.resize(cap);
        type_.resize(cap);
        lst_output out{flat_.data(), flat_.size(), len_.data(), seed_.data(), type_.data(), cap, tco, hco};
        if (lst_batch_get_output(ev_, 0, 1, &out) >= 0)
          break;
        if (tco[1] <= cap)
          throw std::runtime_error(lst_last_error());
        cap = static_cast<size_t>(tco[1]);
      }
      const size_t n = static_cast<size_t>(tco[1]);
      out_tc_hitIdxs_.assign(n, {});
      size_t k = 0;
      for (size_t i = 0; i < n; ++i) {
        out_tc_hitIdxs_[i].assign(flat_.begin() + k, flat_.begin() + k + len_[i]);
        k += len_[i];
      }
      out_tc_len_.assign(len_.begin(), len_.begin() + n);
      out_tc_seedIdx_.assign(seed_.begin(), seed_.begin() + n);
      out_tc_trackCandidateType_.assign(type_.begin(), type_.begin() + n);
    }
    std::vector<std::vector<unsigned int>> hits() { return out_tc_hitIdxs_; }
    std::vector<unsigned int> len() { return out_tc_len_; }
    std::vector<int> seedIdx() { return out_tc_seedIdx_; }
    std::vector<short> trackCandidateType() { return out_tc_trackCandidateType_; }

  private:
    lst_es* es_ = nullptr;
    std::shared_ptr<lst_es> esOwner_;
    lst_event* ev_ = nullptr;
    std::vector<uint32_t> flat_, len_;
    std::vector<int32_t> seed_;
    std::vector<int16_t> type_;
    std::vector<std::vector<unsigned int>> out_tc_hitIdxs_;
    std::vector<unsigned int> out_tc_len_;
    std::vector<int> out_tc_seedIdx_;
    std::vector<short> out_tc_trackCandidateType_;
  };

}  // namespace SDL

#endif  // LST_SDL_HPP
