// C entry points around the LST reference CPU backend (SDL::Event<Acc>), built
// from the unmodified reference sources against the serial Alpaka shim in
// ./shim.  Test infrastructure only: the parity tests, the golden-fixture
// generator and the reference arm of bench.py load the resulting library
// (oracle/_ref/liblstref_*.so).  Nothing in the product links it.
//
// The reference keeps its device buffers private (SDL/Event.h:31-98); the
// field accessor below reads them directly so that every array of every object
// type can be compared, not only the subset the public getters copy
// (SDL/Event.cc:1489-1814).
#include <algorithm>
#include <array>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

// Standard headers are included first so that only the reference's own class
// declarations see the access-specifier override below.
#define private public
#include "Event.h"
#include "LST.h"
#undef private

namespace {
  struct RefES {
    std::unique_ptr<SDL::LSTESHostData<SDL::Dev>> host;
    std::unique_ptr<SDL::LSTESDeviceData<SDL::Dev>> dev;
  };
  struct RefEvent {
    SDL::QueueAcc queue;
    SDL::Event<SDL::Acc> event;
    RefEvent(RefES* es) : queue(SDL::Dev{}), event(false, queue, es->dev.get()) {}
  };

  struct FieldRef {
    const void* ptr = nullptr;
    long long n = 0;
    int size = 0;
  };

  template <typename TBuf>
  FieldRef fieldOf(TBuf const& b) {
    FieldRef f;
    f.ptr = b.data();
    f.n = static_cast<long long>(b.size());
    f.size = static_cast<int>(sizeof(*b.data()));
    return f;
  }

#define LSTREF_F(prefix, obj, name) \
  if (key == prefix #name)          \
    return fieldOf((obj).name##_buf);

  FieldRef lookup(RefEvent* e, std::string const& key) {
    auto& ev = e->event;
    auto const* mods = ev.modulesBuffers_.get();
    if (mods) {
      LSTREF_F("modules.", *mods, detIds)
      LSTREF_F("modules.", *mods, moduleMap)
      LSTREF_F("modules.", *mods, mapdetId)
      LSTREF_F("modules.", *mods, mapIdx)
      LSTREF_F("modules.", *mods, nConnectedModules)
      LSTREF_F("modules.", *mods, drdzs)
      LSTREF_F("modules.", *mods, dxdys)
      LSTREF_F("modules.", *mods, partnerModuleIndices)
      LSTREF_F("modules.", *mods, layers)
      LSTREF_F("modules.", *mods, rings)
      LSTREF_F("modules.", *mods, modules)
      LSTREF_F("modules.", *mods, rods)
      LSTREF_F("modules.", *mods, subdets)
      LSTREF_F("modules.", *mods, sides)
      LSTREF_F("modules.", *mods, eta)
      LSTREF_F("modules.", *mods, r)
      LSTREF_F("modules.", *mods, isInverted)
      LSTREF_F("modules.", *mods, isLower)
      LSTREF_F("modules.", *mods, isAnchor)
      LSTREF_F("modules.", *mods, moduleType)
      LSTREF_F("modules.", *mods, moduleLayerType)
      LSTREF_F("modules.", *mods, sdlLayers)
      LSTREF_F("modules.", *mods, connectedPixels)
    }
    if (key.rfind("pixelmap.", 0) == 0) {
      auto const* pm = ev.pixelMapping_.get();
      auto vec = [](std::vector<unsigned int> const& v) {
        FieldRef f;
        f.ptr = v.data();
        f.n = static_cast<long long>(v.size());
        f.size = 4;
        return f;
      };
      if (key == "pixelmap.connectedPixelsIndex")
        return vec(pm->connectedPixelsIndex);
      if (key == "pixelmap.connectedPixelsSizes")
        return vec(pm->connectedPixelsSizes);
      if (key == "pixelmap.connectedPixelsIndexPos")
        return vec(pm->connectedPixelsIndexPos);
      if (key == "pixelmap.connectedPixelsSizesPos")
        return vec(pm->connectedPixelsSizesPos);
      if (key == "pixelmap.connectedPixelsIndexNeg")
        return vec(pm->connectedPixelsIndexNeg);
      if (key == "pixelmap.connectedPixelsSizesNeg")
        return vec(pm->connectedPixelsSizesNeg);
    }
    if (ev.endcapGeometry_) {
      LSTREF_F("endcap.", *ev.endcapGeometry_, geoMapDetId)
      LSTREF_F("endcap.", *ev.endcapGeometry_, geoMapPhi)
    }
    if (auto* b = ev.hitsBuffers; ev.hitsInGPU && b) {
      LSTREF_F("hits.", *b, nHits)
      LSTREF_F("hits.", *b, xs)
      LSTREF_F("hits.", *b, ys)
      LSTREF_F("hits.", *b, zs)
      LSTREF_F("hits.", *b, moduleIndices)
      LSTREF_F("hits.", *b, idxs)
      LSTREF_F("hits.", *b, detid)
      LSTREF_F("hits.", *b, rts)
      LSTREF_F("hits.", *b, phis)
      LSTREF_F("hits.", *b, etas)
      LSTREF_F("hits.", *b, highEdgeXs)
      LSTREF_F("hits.", *b, highEdgeYs)
      LSTREF_F("hits.", *b, lowEdgeXs)
      LSTREF_F("hits.", *b, lowEdgeYs)
      LSTREF_F("hits.", *b, hitRanges)
      LSTREF_F("hits.", *b, hitRangesLower)
      LSTREF_F("hits.", *b, hitRangesUpper)
      LSTREF_F("hits.", *b, hitRangesnLower)
      LSTREF_F("hits.", *b, hitRangesnUpper)
    }
    if (auto* b = ev.rangesBuffers; ev.rangesInGPU && b) {
      LSTREF_F("ranges.", *b, mdRanges)
      LSTREF_F("ranges.", *b, segmentRanges)
      LSTREF_F("ranges.", *b, tripletRanges)
      LSTREF_F("ranges.", *b, quintupletRanges)
      LSTREF_F("ranges.", *b, nEligibleT5Modules)
      LSTREF_F("ranges.", *b, indicesOfEligibleT5Modules)
      LSTREF_F("ranges.", *b, quintupletModuleIndices)
      LSTREF_F("ranges.", *b, quintupletModuleOccupancy)
      LSTREF_F("ranges.", *b, miniDoubletModuleIndices)
      LSTREF_F("ranges.", *b, miniDoubletModuleOccupancy)
      LSTREF_F("ranges.", *b, segmentModuleIndices)
      LSTREF_F("ranges.", *b, segmentModuleOccupancy)
      LSTREF_F("ranges.", *b, tripletModuleIndices)
      LSTREF_F("ranges.", *b, tripletModuleOccupancy)
      LSTREF_F("ranges.", *b, device_nTotalMDs)
      LSTREF_F("ranges.", *b, device_nTotalSegs)
      LSTREF_F("ranges.", *b, device_nTotalTrips)
      LSTREF_F("ranges.", *b, device_nTotalQuints)
    }
    if (auto* b = ev.miniDoubletsBuffers; ev.mdsInGPU && b) {
      LSTREF_F("md.", *b, nMemoryLocations)
      LSTREF_F("md.", *b, anchorHitIndices)
      LSTREF_F("md.", *b, outerHitIndices)
      LSTREF_F("md.", *b, moduleIndices)
      LSTREF_F("md.", *b, nMDs)
      LSTREF_F("md.", *b, totOccupancyMDs)
      LSTREF_F("md.", *b, dphichanges)
      LSTREF_F("md.", *b, dzs)
      LSTREF_F("md.", *b, dphis)
      LSTREF_F("md.", *b, shiftedXs)
      LSTREF_F("md.", *b, shiftedYs)
      LSTREF_F("md.", *b, shiftedZs)
      LSTREF_F("md.", *b, noShiftedDzs)
      LSTREF_F("md.", *b, noShiftedDphis)
      LSTREF_F("md.", *b, noShiftedDphiChanges)
      LSTREF_F("md.", *b, anchorX)
      LSTREF_F("md.", *b, anchorY)
      LSTREF_F("md.", *b, anchorZ)
      LSTREF_F("md.", *b, anchorRt)
      LSTREF_F("md.", *b, anchorPhi)
      LSTREF_F("md.", *b, anchorEta)
      LSTREF_F("md.", *b, anchorHighEdgeX)
      LSTREF_F("md.", *b, anchorHighEdgeY)
      LSTREF_F("md.", *b, anchorLowEdgeX)
      LSTREF_F("md.", *b, anchorLowEdgeY)
      LSTREF_F("md.", *b, anchorLowEdgePhi)
      LSTREF_F("md.", *b, anchorHighEdgePhi)
      LSTREF_F("md.", *b, outerX)
      LSTREF_F("md.", *b, outerY)
      LSTREF_F("md.", *b, outerZ)
      LSTREF_F("md.", *b, outerRt)
      LSTREF_F("md.", *b, outerPhi)
      LSTREF_F("md.", *b, outerEta)
      LSTREF_F("md.", *b, outerHighEdgeX)
      LSTREF_F("md.", *b, outerHighEdgeY)
      LSTREF_F("md.", *b, outerLowEdgeX)
      LSTREF_F("md.", *b, outerLowEdgeY)
    }
    if (auto* b = ev.segmentsBuffers; ev.segmentsInGPU && b) {
      LSTREF_F("ls.", *b, dPhis)
      LSTREF_F("ls.", *b, dPhiMins)
      LSTREF_F("ls.", *b, dPhiMaxs)
      LSTREF_F("ls.", *b, dPhiChanges)
      LSTREF_F("ls.", *b, dPhiChangeMins)
      LSTREF_F("ls.", *b, dPhiChangeMaxs)
      LSTREF_F("ls.", *b, innerLowerModuleIndices)
      LSTREF_F("ls.", *b, outerLowerModuleIndices)
      LSTREF_F("ls.", *b, seedIdx)
      LSTREF_F("ls.", *b, mdIndices)
      LSTREF_F("ls.", *b, nMemoryLocations)
      LSTREF_F("ls.", *b, innerMiniDoubletAnchorHitIndices)
      LSTREF_F("ls.", *b, outerMiniDoubletAnchorHitIndices)
      LSTREF_F("ls.", *b, charge)
      LSTREF_F("ls.", *b, superbin)
      LSTREF_F("ls.", *b, nSegments)
      LSTREF_F("ls.", *b, totOccupancySegments)
      LSTREF_F("ls.", *b, pLSHitsIdxs)
      LSTREF_F("ls.", *b, pixelType)
      LSTREF_F("ls.", *b, isQuad)
      LSTREF_F("ls.", *b, isDup)
      LSTREF_F("ls.", *b, partOfPT5)
      LSTREF_F("ls.", *b, ptIn)
      LSTREF_F("ls.", *b, ptErr)
      LSTREF_F("ls.", *b, px)
      LSTREF_F("ls.", *b, py)
      LSTREF_F("ls.", *b, pz)
      LSTREF_F("ls.", *b, etaErr)
      LSTREF_F("ls.", *b, eta)
      LSTREF_F("ls.", *b, phi)
      LSTREF_F("ls.", *b, score)
      LSTREF_F("ls.", *b, circleCenterX)
      LSTREF_F("ls.", *b, circleCenterY)
      LSTREF_F("ls.", *b, circleRadius)
    }
    if (auto* b = ev.tripletsBuffers; ev.tripletsInGPU && b) {
      LSTREF_F("t3.", *b, segmentIndices)
      LSTREF_F("t3.", *b, lowerModuleIndices)
      LSTREF_F("t3.", *b, nTriplets)
      LSTREF_F("t3.", *b, totOccupancyTriplets)
      LSTREF_F("t3.", *b, nMemoryLocations)
      LSTREF_F("t3.", *b, logicalLayers)
      LSTREF_F("t3.", *b, hitIndices)
      LSTREF_F("t3.", *b, betaIn)
      LSTREF_F("t3.", *b, circleRadius)
      LSTREF_F("t3.", *b, circleCenterX)
      LSTREF_F("t3.", *b, circleCenterY)
      LSTREF_F("t3.", *b, partOfPT5)
      LSTREF_F("t3.", *b, partOfT5)
      LSTREF_F("t3.", *b, partOfPT3)
    }
    if (auto* b = ev.quintupletsBuffers; ev.quintupletsInGPU && b) {
      LSTREF_F("t5.", *b, tripletIndices)
      LSTREF_F("t5.", *b, lowerModuleIndices)
      LSTREF_F("t5.", *b, nQuintuplets)
      LSTREF_F("t5.", *b, totOccupancyQuintuplets)
      LSTREF_F("t5.", *b, nMemoryLocations)
      LSTREF_F("t5.", *b, innerRadius)
      LSTREF_F("t5.", *b, bridgeRadius)
      LSTREF_F("t5.", *b, outerRadius)
      LSTREF_F("t5.", *b, pt)
      LSTREF_F("t5.", *b, eta)
      LSTREF_F("t5.", *b, phi)
      LSTREF_F("t5.", *b, score_rphisum)
      LSTREF_F("t5.", *b, layer)
      LSTREF_F("t5.", *b, isDup)
      LSTREF_F("t5.", *b, TightCutFlag)
      LSTREF_F("t5.", *b, partOfPT5)
      LSTREF_F("t5.", *b, regressionRadius)
      LSTREF_F("t5.", *b, regressionG)
      LSTREF_F("t5.", *b, regressionF)
      LSTREF_F("t5.", *b, logicalLayers)
      LSTREF_F("t5.", *b, hitIndices)
      LSTREF_F("t5.", *b, rzChiSquared)
      LSTREF_F("t5.", *b, chiSquared)
      LSTREF_F("t5.", *b, nonAnchorChiSquared)
    }
    if (auto* b = ev.pixelTripletsBuffers; ev.pixelTripletsInGPU && b) {
      LSTREF_F("pt3.", *b, pixelSegmentIndices)
      LSTREF_F("pt3.", *b, tripletIndices)
      LSTREF_F("pt3.", *b, nPixelTriplets)
      LSTREF_F("pt3.", *b, totOccupancyPixelTriplets)
      LSTREF_F("pt3.", *b, pixelRadius)
      LSTREF_F("pt3.", *b, tripletRadius)
      LSTREF_F("pt3.", *b, pt)
      LSTREF_F("pt3.", *b, eta)
      LSTREF_F("pt3.", *b, phi)
      LSTREF_F("pt3.", *b, eta_pix)
      LSTREF_F("pt3.", *b, phi_pix)
      LSTREF_F("pt3.", *b, score)
      LSTREF_F("pt3.", *b, isDup)
      LSTREF_F("pt3.", *b, partOfPT5)
      LSTREF_F("pt3.", *b, logicalLayers)
      LSTREF_F("pt3.", *b, hitIndices)
      LSTREF_F("pt3.", *b, lowerModuleIndices)
      LSTREF_F("pt3.", *b, centerX)
      LSTREF_F("pt3.", *b, centerY)
      LSTREF_F("pt3.", *b, pixelRadiusError)
      LSTREF_F("pt3.", *b, rPhiChiSquared)
      LSTREF_F("pt3.", *b, rPhiChiSquaredInwards)
      LSTREF_F("pt3.", *b, rzChiSquared)
    }
    if (auto* b = ev.pixelQuintupletsBuffers; ev.pixelQuintupletsInGPU && b) {
      LSTREF_F("pt5.", *b, pixelIndices)
      LSTREF_F("pt5.", *b, T5Indices)
      LSTREF_F("pt5.", *b, nPixelQuintuplets)
      LSTREF_F("pt5.", *b, totOccupancyPixelQuintuplets)
      LSTREF_F("pt5.", *b, isDup)
      LSTREF_F("pt5.", *b, score)
      LSTREF_F("pt5.", *b, eta)
      LSTREF_F("pt5.", *b, phi)
      LSTREF_F("pt5.", *b, logicalLayers)
      LSTREF_F("pt5.", *b, hitIndices)
      LSTREF_F("pt5.", *b, lowerModuleIndices)
      LSTREF_F("pt5.", *b, pixelRadius)
      LSTREF_F("pt5.", *b, quintupletRadius)
      LSTREF_F("pt5.", *b, centerX)
      LSTREF_F("pt5.", *b, centerY)
      LSTREF_F("pt5.", *b, rzChiSquared)
      LSTREF_F("pt5.", *b, rPhiChiSquared)
      LSTREF_F("pt5.", *b, rPhiChiSquaredInwards)
    }
    if (auto* b = ev.trackCandidatesBuffers; ev.trackCandidatesInGPU && b) {
      LSTREF_F("tc.", *b, trackCandidateType)
      LSTREF_F("tc.", *b, directObjectIndices)
      LSTREF_F("tc.", *b, objectIndices)
      LSTREF_F("tc.", *b, nTrackCandidates)
      LSTREF_F("tc.", *b, nTrackCandidatespT3)
      LSTREF_F("tc.", *b, nTrackCandidatespT5)
      LSTREF_F("tc.", *b, nTrackCandidatespLS)
      LSTREF_F("tc.", *b, nTrackCandidatesT5)
      LSTREF_F("tc.", *b, logicalLayers)
      LSTREF_F("tc.", *b, hitIndices)
      LSTREF_F("tc.", *b, pixelSeedIndex)
      LSTREF_F("tc.", *b, lowerModuleIndices)
      LSTREF_F("tc.", *b, centerX)
      LSTREF_F("tc.", *b, centerY)
      LSTREF_F("tc.", *b, radius)
    }
    return FieldRef{};
  }
#undef LSTREF_F
}  // namespace

extern "C" {

// Loads the event setup from <lst_base>/data/OT800_IT615_pt0.8 (the reference
// reads $LST_BASE, SDL/LSTESData.cc:14-30).  Returns nullptr on failure.
void* lstref_es_load(const char* lst_base) {
  try {
    setenv("LST_BASE", lst_base, 1);
    auto* es = new RefES();
    es->host = SDL::loadAndFillESHost();
    SDL::QueueAcc queue(SDL::Dev{});
    es->dev = SDL::loadAndFillESDevice(queue, es->host.get());
    return es;
  } catch (...) {
    return nullptr;
  }
}

void lstref_es_free(void* es) { delete static_cast<RefES*>(es); }

unsigned int lstref_es_counts(void* es, unsigned int* nModules, unsigned int* nLowerModules) {
  auto* e = static_cast<RefES*>(es);
  *nModules = e->dev->nModules;
  *nLowerModules = e->dev->nLowerModules;
  return e->dev->nPixels;
}

void* lstref_event_create(void* es) { return new RefEvent(static_cast<RefES*>(es)); }

void lstref_event_destroy(void* ev) {
  auto* e = static_cast<RefEvent*>(ev);
  e->event.resetEvent();
  delete e;
}

void lstref_event_reset(void* ev) { static_cast<RefEvent*>(ev)->event.resetEvent(); }

void lstref_event_add_hits(void* ev,
                           unsigned int n,
                           const float* x,
                           const float* y,
                           const float* z,
                           const unsigned int* detId,
                           const unsigned int* idx) {
  auto* e = static_cast<RefEvent*>(ev);
  e->event.addHitToEvent(std::vector<float>(x, x + n),
                         std::vector<float>(y, y + n),
                         std::vector<float>(z, z + n),
                         std::vector<unsigned int>(detId, detId + n),
                         std::vector<unsigned int>(idx, idx + n));
}

void lstref_event_add_pixel_segments(void* ev,
                                     unsigned int n,
                                     const unsigned int* hitIndices0,
                                     const unsigned int* hitIndices1,
                                     const unsigned int* hitIndices2,
                                     const unsigned int* hitIndices3,
                                     const float* dPhiChange,
                                     const float* ptIn,
                                     const float* ptErr,
                                     const float* px,
                                     const float* py,
                                     const float* pz,
                                     const float* eta,
                                     const float* etaErr,
                                     const float* phi,
                                     const int* charge,
                                     const unsigned int* seedIdx,
                                     const int* superbin,
                                     const int8_t* pixelType,
                                     const char* isQuad) {
  auto* e = static_cast<RefEvent*>(ev);
  auto u = [n](const unsigned int* p) { return std::vector<unsigned int>(p, p + n); };
  auto f = [n](const float* p) { return std::vector<float>(p, p + n); };
  e->event.addPixelSegmentToEvent(u(hitIndices0),
                                  u(hitIndices1),
                                  u(hitIndices2),
                                  u(hitIndices3),
                                  f(dPhiChange),
                                  f(ptIn),
                                  f(ptErr),
                                  f(px),
                                  f(py),
                                  f(pz),
                                  f(eta),
                                  f(etaErr),
                                  f(phi),
                                  std::vector<int>(charge, charge + n),
                                  u(seedIdx),
                                  std::vector<int>(superbin, superbin + n),
                                  std::vector<int8_t>(pixelType, pixelType + n),
                                  std::vector<char>(isQuad, isQuad + n));
}

// Runs one stage of the chain, in the order bin/sdl.cc:451-458 calls them:
// 1 createMiniDoublets, 2 createSegmentsWithModuleMap, 3 createTriplets,
// 4 createQuintuplets, 5 pixelLineSegmentCleaning, 6 createPixelQuintuplets,
// 7 createPixelTriplets, 8 createTrackCandidates.
int lstref_event_run_stage(void* ev, int stage) {
  auto& event = static_cast<RefEvent*>(ev)->event;
  switch (stage) {
    case 1:
      event.createMiniDoublets();
      return 0;
    case 2:
      event.createSegmentsWithModuleMap();
      return 0;
    case 3:
      event.createTriplets();
      return 0;
    case 4:
      event.createQuintuplets();
      return 0;
    case 5:
      event.pixelLineSegmentCleaning();
      return 0;
    case 6:
      event.createPixelQuintuplets();
      return 0;
    case 7:
      event.createPixelTriplets();
      return 0;
    case 8:
      event.createTrackCandidates();
      return 0;
    default:
      return -1;
  }
}

// ---------------------------------------------------------------- SDL::LST
// The CMSSW entry point (SDL/LST.h:25-111).  Seeds come as 13 float arrays in
// LST::run's argument order (see_px .. see_stateTrajGlbPz), see_q, and
// see_hitIdx flattened as offsets (n_seeds + 1) plus values.
namespace {
  struct RefLSTRun {
    SDL::LST<SDL::Acc> lst;
    std::vector<unsigned int> flatHits;  // out_tc_hitIdxs_ concatenated
  };

  struct SeedVectors {
    std::vector<float> f[13];
    std::vector<int> q;
    std::vector<std::vector<int>> hitIdx;
    std::vector<unsigned int> detId;
    std::vector<float> x, y, z;
  };

  SeedVectors seedVectors(unsigned int nSeeds,
                          const float* const* f13,
                          const int* q,
                          const unsigned int* hitOff,
                          const int* hitIdx,
                          unsigned int nPh2,
                          const unsigned int* detId,
                          const float* x,
                          const float* y,
                          const float* z) {
    SeedVectors v;
    for (int k = 0; k < 13; ++k)
      v.f[k].assign(f13[k], f13[k] + nSeeds);
    v.q.assign(q, q + nSeeds);
    v.hitIdx.resize(nSeeds);
    for (unsigned int i = 0; i < nSeeds; ++i)
      v.hitIdx[i].assign(hitIdx + hitOff[i], hitIdx + hitOff[i + 1]);
    v.detId.assign(detId, detId + nPh2);
    v.x.assign(x, x + nPh2);
    v.y.assign(y, y + nPh2);
    v.z.assign(z, z + nPh2);
    return v;
  }
}  // namespace

void* lstref_lst_create() { return new RefLSTRun(); }

void lstref_lst_destroy(void* l) { delete static_cast<RefLSTRun*>(l); }

// LST::prepareInput (SDL/LST.cc:175-365) alone; its results are read with
// lstref_lst_array ("in_trkX_", "in_hitIndices_vec0_", ...).
void lstref_lst_prepare(void* l,
                        unsigned int nSeeds,
                        const float* const* f13,
                        const int* q,
                        const unsigned int* hitOff,
                        const int* hitIdx,
                        unsigned int nPh2,
                        const unsigned int* detId,
                        const float* x,
                        const float* y,
                        const float* z) {
  auto v = seedVectors(nSeeds, f13, q, hitOff, hitIdx, nPh2, detId, x, y, z);
  static_cast<RefLSTRun*>(l)->lst.prepareInput(v.f[0], v.f[1], v.f[2], v.f[3], v.f[4], v.f[5], v.f[6], v.f[7],
                                               v.f[8], v.f[9], v.f[10], v.f[11], v.f[12], v.q, v.hitIdx, v.detId,
                                               v.x, v.y, v.z);
}

// LST::run (SDL/LST.cc:12-161): conversion, the whole chain on a fresh Event
// and getOutput; the outputs are read with lstref_lst_array ("out_tc_len_",
// "out_tc_seedIdx_", "out_tc_trackCandidateType_", and "out_tc_hitIdxs_" as
// the per-candidate lists concatenated).
void lstref_lst_run(void* l,
                    void* es,
                    unsigned int nSeeds,
                    const float* const* f13,
                    const int* q,
                    const unsigned int* hitOff,
                    const int* hitIdx,
                    unsigned int nPh2,
                    const unsigned int* detId,
                    const float* x,
                    const float* y,
                    const float* z) {
  auto* r = static_cast<RefLSTRun*>(l);
  auto v = seedVectors(nSeeds, f13, q, hitOff, hitIdx, nPh2, detId, x, y, z);
  SDL::QueueAcc queue(SDL::Dev{});
  r->lst.run(queue, false, static_cast<RefES*>(es)->dev.get(), v.f[0], v.f[1], v.f[2], v.f[3], v.f[4], v.f[5],
             v.f[6], v.f[7], v.f[8], v.f[9], v.f[10], v.f[11], v.f[12], v.q, v.hitIdx, v.detId, v.x, v.y, v.z);
  r->flatHits.clear();
  for (auto const& h : r->lst.out_tc_hitIdxs_)
    r->flatHits.insert(r->flatHits.end(), h.begin(), h.end());
}

const void* lstref_lst_array(void* l, const char* name, long long* n, int* elem_size) {
  auto* r = static_cast<RefLSTRun*>(l);
  auto& L = r->lst;
  std::string key(name);
  const void* ptr = nullptr;
  auto take = [&](auto const& vec) {
    ptr = vec.data();
    *n = static_cast<long long>(vec.size());
    *elem_size = static_cast<int>(sizeof(vec[0]));
  };
  *n = 0;
  *elem_size = 0;
#define LSTREF_V(member) \
  if (key == #member)    \
    take(L.member);
  LSTREF_V(in_trkX_)
  LSTREF_V(in_trkY_)
  LSTREF_V(in_trkZ_)
  LSTREF_V(in_hitId_)
  LSTREF_V(in_hitIdxs_)
  LSTREF_V(in_hitIndices_vec0_)
  LSTREF_V(in_hitIndices_vec1_)
  LSTREF_V(in_hitIndices_vec2_)
  LSTREF_V(in_hitIndices_vec3_)
  LSTREF_V(in_deltaPhi_vec_)
  LSTREF_V(in_ptIn_vec_)
  LSTREF_V(in_ptErr_vec_)
  LSTREF_V(in_px_vec_)
  LSTREF_V(in_py_vec_)
  LSTREF_V(in_pz_vec_)
  LSTREF_V(in_eta_vec_)
  LSTREF_V(in_etaErr_vec_)
  LSTREF_V(in_phi_vec_)
  LSTREF_V(in_charge_vec_)
  LSTREF_V(in_seedIdx_vec_)
  LSTREF_V(in_superbin_vec_)
  LSTREF_V(in_pixelType_vec_)
  LSTREF_V(in_isQuad_vec_)
  LSTREF_V(out_tc_len_)
  LSTREF_V(out_tc_seedIdx_)
  LSTREF_V(out_tc_trackCandidateType_)
#undef LSTREF_V
  if (key == "out_tc_hitIdxs_")
    take(r->flatHits);
  return ptr;
}

// Returns a pointer to the named internal array (e.g. "md.anchorHitIndices"),
// its element count and element size, or nullptr if the array does not exist
// (yet) for this event.
const void* lstref_event_field(void* ev, const char* name, long long* n, int* elem_size) {
  FieldRef f = lookup(static_cast<RefEvent*>(ev), name);
  *n = f.n;
  *elem_size = f.size;
  return f.ptr;
}

}  // extern "C"
