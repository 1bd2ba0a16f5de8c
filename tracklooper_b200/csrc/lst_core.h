// Core definitions shared by the CUDA kernels of the LST object-building chain:
// compile-target macros, the reference's constants and enumerations, the
// floating-point binding of the transcendental functions, the geometric helpers
// (phi, deltaPhi, ...) and the structure-of-arrays views of every object store.
//
// Floating-point contract.  Every arithmetic expression in the cut functions
// keeps the operand types and evaluation order of the reference
// (SDL/*.h), and the library is compiled with --fmad=false and IEEE division
// and square root, so +, -, *, / and sqrt round exactly as the reference's
// strict CPU build does.  The float transcendentals (sin, cos, tan, asin, acos,
// atan, atan2, sinh, acosh, exp, log) are evaluated as float(f(double(x))):
// the double result is within a few double ulps of the exact value on every
// platform, so the rounded float agrees across CPU and GPU except when the
// exact value lies within ~2^-29 relative of a float rounding boundary.
#pragma once

#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define LST_HD __host__ __device__ __forceinline__
#define LST_DEV __device__ __forceinline__
// The large cut algorithms are inlined into their kernels.  Out of line, each
// call saves and restores the caller's live registers through local memory,
// which cost more than the instruction-cache misses of the larger inlined
// code once candidates reach them through the sorted pre-selection queues.
// The double-precision math routines (LST_HD_MATH) stay out of line.
#define LST_HD_BIG __host__ __device__ __forceinline__
#else
#define LST_HD inline
#define LST_DEV inline
#define LST_HD_BIG inline
#endif

namespace lst {

  // ------------------------------------------------------------------ enums
  // Values as in SDL/Module.h:13-19.
  enum SubDet : short { InnerPixel = 0, Barrel = 5, Endcap = 4 };
  enum Side : short { NegZ = 1, PosZ = 2, Center = 3 };
  enum ModuleType : uint8_t { PS = 0, TwoS = 1, PixelModule = 2 };
  enum ModuleLayerType : uint8_t { Pixel = 0, Strip = 1, InnerPixelLayer = 2 };

  // ------------------------------------------------------------- capacities
  // SDL/Constants.h:107-121.
  // Connected modules per module in the module map, and pixel-map modules per
  // pLS superbin.  The reference's rows hold 40 (SDL/Constants.h:107), which
  // the pt0.8 maps fill at most; the pt0.6 maps list up to 68 for 1328
  // modules, more than the reference's rows hold (SDL/ModuleMethods.h:127-134
  // would write past them), so the rows here hold 80.  Row length changes no
  // object of the pt0.8 geometry.
  constexpr unsigned int kMaxConnectedModules = 80;
  constexpr unsigned int kMaxPixelSegments = 50000;
  constexpr unsigned int kMaxPixelMDs = 2 * kMaxPixelSegments;
  constexpr unsigned int kMaxPixelTriplets = 5000;
  constexpr unsigned int kMaxPixelQuintuplets = 15000;
  constexpr unsigned int kMaxPixelTrackCandidates = 30000;
  constexpr unsigned int kMaxNonPixelTrackCandidates = 1000;
  constexpr unsigned int kMaxTrackCandidates = kMaxPixelTrackCandidates + kMaxNonPixelTrackCandidates;
  constexpr unsigned int kSizeSuperbins = 45000;

  // ------------------------------------------------------ physics constants
  // SDL/Constants.h:123-139; initialised from the same double expressions.
  constexpr float k2Rinv1GeVf = (2.99792458e-3 * 3.8) / 2;
  constexpr float kR1GeVf = 1. / (2.99792458e-3 * 3.8);
  constexpr float kSinAlphaMax = 0.95;
  // The transverse-momentum cut the module and pixel maps are built for
  // (SDL/Constants.h:102-105 sets it at compile time, PT_CUT, default 0.8
  // GeV); here it is a property of the loaded geometry, Modules::ptCut.
  constexpr float kPtCut = 0.8f;
  constexpr float kDeltaZLum = 15.0;
  constexpr float kPixelPSZpitch = 0.15;
  constexpr float kStrip2SZpitch = 5.0;
  constexpr float kPtBetaMax = 7.0;
  constexpr float kMagneticField = 3.8112;
  constexpr float kInf = 123456789;  // the reference's stand-in for infinity
  constexpr float kPi = float(M_PI);

  // T5 DNN working point used for T5 building (SDL/Constants.h:145).
  constexpr float kT5DnnWP = 0.6177366f;

  // --------------------------------------------------- math binding (see top)
  // One out-of-line copy of each double-precision routine on the device: the
  // cut algorithms call them from dozens of sites, and an inlined copy per
  // site multiplies the code the diverging warps of one SM fetch.
#if defined(__CUDACC__)
#define LST_HD_MATH static __host__ __device__ __noinline__  // one copy per translation unit
#else
#define LST_HD_MATH inline
#endif
  // A host build that evaluates these headers in another arithmetic (the
  // cut-flip tracer under oracle/trace/) defines LST_MATH_BINDING_PROVIDED and
  // supplies the functions of this block itself.
#if !defined(LST_MATH_BINDING_PROVIDED)
  LST_HD_MATH float fsin(float x) { return static_cast<float>(::sin(static_cast<double>(x))); }
  LST_HD_MATH float fcos(float x) { return static_cast<float>(::cos(static_cast<double>(x))); }
  LST_HD_MATH float ftan(float x) { return static_cast<float>(::tan(static_cast<double>(x))); }
  LST_HD_MATH float fasin(float x) { return static_cast<float>(::asin(static_cast<double>(x))); }
  LST_HD_MATH float facos(float x) { return static_cast<float>(::acos(static_cast<double>(x))); }
  LST_HD_MATH float fatan(float x) { return static_cast<float>(::atan(static_cast<double>(x))); }
  LST_HD_MATH float fsinh(float x) { return static_cast<float>(::sinh(static_cast<double>(x))); }
  LST_HD_MATH float facosh(float x) { return static_cast<float>(::acosh(static_cast<double>(x))); }
  LST_HD_MATH float fexp(float x) { return static_cast<float>(::exp(static_cast<double>(x))); }
  LST_HD_MATH float flog(float x) { return static_cast<float>(::log(static_cast<double>(x))); }
  LST_HD_MATH float fatan2(float y, float x) {
    return static_cast<float>(::atan2(static_cast<double>(y), static_cast<double>(x)));
  }
  // Exact operations.
  LST_HD float fabs_(float x) { return ::fabsf(x); }
  LST_HD double fabs_(double x) { return ::fabs(x); }
  LST_HD float fmin_(float a, float b) { return ::fminf(a, b); }
  LST_HD float fmax_(float a, float b) { return ::fmaxf(a, b); }
  LST_HD double fmin_(float a, double b) { return ::fmin(static_cast<double>(a), b); }
  LST_HD double fmax_(float a, double b) { return ::fmax(static_cast<double>(a), b); }
  LST_HD float fsqrt(float x) { return ::sqrtf(x); }
  LST_HD double dsqrt(double x) { return ::sqrt(x); }
  LST_HD bool fisnan(float x) { return x != x; }
  LST_HD float fround_(float x) { return ::roundf(x); }
#endif  // LST_MATH_BINDING_PROVIDED

  // ------------------------------------------------------ geometric helpers
  // SDL/Hit.h:111-192.
  LST_HD float log10_(float val) {
    constexpr float ln10 = 2.302585093f;
    return flog(val) / ln10;
  }

  LST_HD float phiMpiPi(float x) {
    if (fabs_(x) <= float(M_PI))
      return x;
    constexpr float o2pi = 1.f / (2.f * float(M_PI));
    float n = fround_(x * o2pi);
    return x - n * float(2.f * float(M_PI));
  }

  LST_HD float phiOf(float x, float y) { return phiMpiPi(float(M_PI) + fatan2(-y, -x)); }

  LST_HD float deltaPhi(float x1, float y1, float x2, float y2) {
    float phi1 = phiOf(x1, y1);
    float phi2 = phiOf(x2, y2);
    return phiMpiPi(phi2 - phi1);
  }

  LST_HD float deltaPhiChange(float x1, float y1, float x2, float y2) { return deltaPhi(x1, y1, x2 - x1, y2 - y1); }

  // deltaPhiChange(x1, y1, x2, y2) with phi1 = phiOf(x1, y1) already known.
  LST_HD float deltaPhiChangeFrom(float phi1, float x1, float y1, float x2, float y2) {
    return phiMpiPi(phiOf(x2 - x1, y2 - y1) - phi1);
  }

  // The reference's sign transfer: |a| with the product of the signs of a and b.
  LST_HD float signTransfer(float a, float b) {
    int sign_a = (a < 0) ? -1 : 1;
    int sign_b = (b < 0) ? -1 : 1;
    return sign_a * sign_b * a;
  }

  LST_HD float wrapDPhi(float phi1, float phi2) {
    float dPhi = phi1 - phi2;
    if (dPhi > float(M_PI)) {
      dPhi -= 2 * float(M_PI);
    } else if (dPhi < -float(M_PI)) {
      dPhi += 2 * float(M_PI);
    }
    return dPhi;
  }

  // Index of search_val in the sorted array data[0, ndata), or -1.
  LST_HD int sortedFind(const unsigned int* data, unsigned int search_val, unsigned int ndata) {
    unsigned int low = 0;
    unsigned int high = ndata - 1;
    while (low <= high) {
      unsigned int mid = (low + high) / 2;
      unsigned int test_val = data[mid];
      if (test_val == search_val)
        return mid;
      else if (test_val > search_val)
        high = mid - 1;
      else
        low = mid + 1;
    }
    return -1;
  }

  // -------------------------------------------------------- object stores
  // Structure-of-arrays views.  Field names follow the reference stores
  // (SDL/Module.h, Hit.h, MiniDoublet.h, Segment.h, Triplet.h, Quintuplet.h,
  // PixelTriplet.h, TrackCandidate.h) so getters can expose them unchanged.

  struct Modules {
    const unsigned int* detIds;
    const uint16_t* moduleMap;
    const unsigned int* mapdetId;
    const uint16_t* mapIdx;
    const uint16_t* nConnectedModules;
    const float* drdzs;
    const float* dxdys;
    const uint16_t* partnerModuleIndices;
    const short* layers;
    const short* rings;
    const short* modules;
    const short* rods;
    const short* subdets;
    const short* sides;
    const float* eta;
    const float* r;
    const uint8_t* isInverted;
    const uint8_t* isLower;
    const uint8_t* isAnchor;
    const uint8_t* moduleType;
    const uint8_t* moduleLayerType;
    const int* sdlLayers;
    const unsigned int* connectedPixels;
    // endcap 2S strip orientation map (SDL/EndcapGeometry.cc:43-70)
    const unsigned int* geoMapDetId;
    const float* geoMapPhi;
    const int* geoMapIndex;  // per module: position of its detId in geoMapDetId, or -1
    unsigned int nEndCapMap;
    uint16_t nModules;
    uint16_t nLowerModules;
    float ptCut;  // the geometry's pt cut (GeV): 0.8 for OT800_IT615_pt0.8, 0.6 for _pt0.6
  };

  struct Hits {
    float* xs;
    float* ys;
    float* zs;
    uint16_t* moduleIndices;
    unsigned int* idxs;
    unsigned int* detid;
    float* rts;
    float* phis;
    float* etas;
    float* highEdgeXs;
    float* highEdgeYs;
    float* lowEdgeXs;
    float* lowEdgeYs;
    int* hitRanges;
    int* hitRangesLower;
    int* hitRangesUpper;
    int8_t* hitRangesnLower;
    int8_t* hitRangesnUpper;
  };

  struct MiniDoublets {
    unsigned int* anchorHitIndices;
    unsigned int* outerHitIndices;
    uint16_t* moduleIndices;
    unsigned int* nMDs;
    unsigned int* totOccupancyMDs;
    float* dphichanges;
    float* dzs;
    float* dphis;
    float* shiftedXs;
    float* shiftedYs;
    float* shiftedZs;
    float* noShiftedDzs;
    float* noShiftedDphis;
    float* noShiftedDphiChanges;
    float* anchorX;
    float* anchorY;
    float* anchorZ;
    float* anchorRt;
    float* anchorPhi;
    float* anchorEta;
    float* anchorHighEdgeX;
    float* anchorHighEdgeY;
    float* anchorLowEdgeX;
    float* anchorLowEdgeY;
    float* anchorLowEdgePhi;
    float* anchorHighEdgePhi;
    float* outerX;
    float* outerY;
    float* outerZ;
    float* outerRt;
    float* outerPhi;
    float* outerEta;
    float* outerHighEdgeX;
    float* outerHighEdgeY;
    float* outerLowEdgeX;
    float* outerLowEdgeY;
    // Derived per mini-doublet from its anchor radius rt (not reference
    // fields): slope = asin(min(rt k / ptCut, sinAlphaMax)), tanSlope =
    // tan(slope), slope3 = asin(min(rt k / 3, sinAlphaMax)).  The cut
    // algorithms evaluate exactly these expressions of a mini-doublet's rt
    // many times over; stored once, they give the same values.
    float* slope;
    float* tanSlope;
    float* slope3;
    // The anchor hit's x, y, z, rt in one 16-byte record: the segment, triplet
    // and pixel kernels gather them together for mini-doublets chosen by index.
    struct MDPos* anchorPos;
    // Everything the segment cuts read of a mini-doublet, in one 48-byte
    // record (three 16-byte loads instead of a dozen scattered ones).
    struct MDRec* rec;
  };

  struct alignas(16) MDPos {
    float x, y, z, rt;
  };

  struct alignas(16) MDRec {
    float x, y, z, rt;                         // anchor hit
    float phi, slope, tanSlope, dphichange;    // anchorPhi, slope, tanSlope, dphichanges
    float dphi, dz, highEdgePhi, lowEdgePhi;   // dphis, dzs, anchorHighEdgePhi, anchorLowEdgePhi
  };

  struct Segments {
    float* dPhis;
    float* dPhiMins;
    float* dPhiMaxs;
    float* dPhiChanges;
    float* dPhiChangeMins;
    float* dPhiChangeMaxs;
    uint16_t* innerLowerModuleIndices;
    uint16_t* outerLowerModuleIndices;
    unsigned int* mdIndices;
    unsigned int* innerMiniDoubletAnchorHitIndices;
    unsigned int* outerMiniDoubletAnchorHitIndices;
    unsigned int* nSegments;
    unsigned int* totOccupancySegments;
    // pixel line segments (indexed by pLS array index 0..nPLS-1)
    unsigned int* seedIdx;
    int* charge;
    int* superbin;
    unsigned int* pLSHitsIdxs;  // 4 per pLS: x, y, z, w
    int8_t* pixelType;
    int8_t* isQuad;
    int8_t* isDup;
    uint8_t* partOfPT5;
    float* ptIn;
    float* ptErr;
    float* px;
    float* py;
    float* pz;
    float* etaErr;
    float* eta;
    float* phi;
    float* score;
    float* circleCenterX;
    float* circleCenterY;
    float* circleRadius;
  };

  struct Triplets {
    unsigned int* segmentIndices;
    uint16_t* lowerModuleIndices;
    unsigned int* nTriplets;
    unsigned int* totOccupancyTriplets;
    uint8_t* logicalLayers;
    unsigned int* hitIndices;
    float* betaIn;
    float* circleRadius;
    float* circleCenterX;
    float* circleCenterY;
    uint8_t* partOfPT5;
    uint8_t* partOfT5;
    uint8_t* partOfPT3;
  };

  struct Quintuplets {
    unsigned int* tripletIndices;
    uint16_t* lowerModuleIndices;
    unsigned int* nQuintuplets;
    unsigned int* totOccupancyQuintuplets;
    float* innerRadius;
    float* bridgeRadius;
    float* outerRadius;
    float* pt;
    float* eta;
    float* phi;
    float* score_rphisum;
    uint8_t* layer;
    int8_t* isDup;
    uint8_t* TightCutFlag;
    uint8_t* partOfPT5;
    float* regressionRadius;
    float* regressionG;
    float* regressionF;
    uint8_t* logicalLayers;
    unsigned int* hitIndices;
    float* rzChiSquared;
    float* chiSquared;
    float* nonAnchorChiSquared;
  };

  struct PixelTriplets {
    unsigned int* pixelSegmentIndices;
    unsigned int* tripletIndices;
    unsigned int* nPixelTriplets;
    unsigned int* totOccupancyPixelTriplets;
    float* pixelRadius;
    float* tripletRadius;
    float* pt;
    float* eta;
    float* phi;
    float* eta_pix;
    float* phi_pix;
    float* score;
    uint8_t* isDup;
    uint8_t* partOfPT5;
    uint8_t* logicalLayers;
    unsigned int* hitIndices;
    uint16_t* lowerModuleIndices;
    float* centerX;
    float* centerY;
    float* pixelRadiusError;
    float* rPhiChiSquared;
    float* rPhiChiSquaredInwards;
    float* rzChiSquared;
  };

  struct PixelQuintuplets {
    unsigned int* pixelIndices;
    unsigned int* T5Indices;
    unsigned int* nPixelQuintuplets;
    unsigned int* totOccupancyPixelQuintuplets;
    uint8_t* isDup;
    float* score;
    float* eta;
    float* phi;
    uint8_t* logicalLayers;
    unsigned int* hitIndices;
    uint16_t* lowerModuleIndices;
    float* pixelRadius;
    float* quintupletRadius;
    float* centerX;
    float* centerY;
    float* rzChiSquared;
    float* rPhiChiSquared;
    float* rPhiChiSquaredInwards;
  };

  struct TrackCandidates {
    short* trackCandidateType;
    unsigned int* directObjectIndices;
    unsigned int* objectIndices;
    unsigned int* nTrackCandidates;
    unsigned int* nTrackCandidatespT3;
    unsigned int* nTrackCandidatespT5;
    unsigned int* nTrackCandidatespLS;
    unsigned int* nTrackCandidatesT5;
    uint8_t* logicalLayers;
    unsigned int* hitIndices;
    int* pixelSeedIndex;
    uint16_t* lowerModuleIndices;
    float* centerX;
    float* centerY;
    float* radius;
  };

  // Per-module offsets and occupancy caps (SDL/Module.h:21-86).
  struct Ranges {
    int* mdRanges;
    int* segmentRanges;
    int* tripletRanges;
    int* quintupletRanges;
    uint16_t* nEligibleT5Modules;
    uint16_t* indicesOfEligibleT5Modules;
    int* quintupletModuleIndices;
    int* quintupletModuleOccupancy;
    int* miniDoubletModuleIndices;
    int* miniDoubletModuleOccupancy;
    int* segmentModuleIndices;
    int* segmentModuleOccupancy;
    int* tripletModuleIndices;
    int* tripletModuleOccupancy;
    unsigned int* device_nTotalMDs;
    unsigned int* device_nTotalSegs;
    unsigned int* device_nTotalTrips;
    unsigned int* device_nTotalQuints;
  };

}  // namespace lst
