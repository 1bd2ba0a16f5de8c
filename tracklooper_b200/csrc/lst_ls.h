// Line-segment (LS) selection: a pair of mini-doublets on module-map-connected
// modules; plus the pixel line segments (pLS) built from pixel seeds.  Cut
// arithmetic follows SDL/Segment.h:264-796 and SDL/Segment.h:392-453,1031-1117.
#pragma once

#include "lst_md.h"

namespace lst {

  // Thresholds of the three alpha (direction) differences
  // (SDL/Segment.h:264-356).
  LST_HD void lsDAlphaThresholds(const Modules& m,
                                 const MiniDoublets& md,
                                 float xIn,
                                 float yIn,
                                 float zIn,
                                 float rtIn,
                                 float xOut,
                                 float yOut,
                                 float zOut,
                                 float rtOut,
                                 uint16_t innerLM,
                                 uint16_t outerLM,
                                 unsigned int innerMD,
                                 unsigned int outerMD,
                                 float* thr) {
    const bool innerBarrel = m.subdets[innerLM] == Barrel;
    const bool outerBarrel = m.subdets[outerLM] == Barrel;
    float sdMuls = innerBarrel ? miniMulsPtScaleBarrel(m.layers[innerLM] - 1) * 3.f / m.ptCut
                               : miniMulsPtScaleEndcap(m.layers[innerLM] - 1) * 3.f / m.ptCut;
    float segmentDr = fsqrt((yOut - yIn) * (yOut - yIn) + (xOut - xIn) * (xOut - xIn));
    const float dAlpha_Bfield = fasin(fmin_(segmentDr * k2Rinv1GeVf / m.ptCut, kSinAlphaMax));
    bool isInnerTilted = innerBarrel and m.sides[innerLM] != Center;
    bool isOuterTilted = outerBarrel and m.sides[outerLM] != Center;
    const float drdzInner = m.drdzs[innerLM];
    const float drdzOuter = m.drdzs[outerLM];
    float innerModuleGapSize = moduleGap(m, innerLM);
    float outerModuleGapSize = moduleGap(m, outerLM);
    const float innerminiTilt =
        isInnerTilted ? (0.5f * kPixelPSZpitch * drdzInner / fsqrt(1.f + drdzInner * drdzInner) / innerModuleGapSize)
                      : 0;
    const float outerminiTilt =
        isOuterTilted ? (0.5f * kPixelPSZpitch * drdzOuter / fsqrt(1.f + drdzOuter * drdzOuter) / outerModuleGapSize)
                      : 0;
    float miniDelta = innerModuleGapSize;
    float sdLumForInnerMini, sdLumForOuterMini;
    if (innerBarrel)
      sdLumForInnerMini = innerminiTilt * dAlpha_Bfield;
    else
      sdLumForInnerMini = md.rec[innerMD].dphi * 15.0f / md.rec[innerMD].dz;
    if (outerBarrel)
      sdLumForOuterMini = outerminiTilt * dAlpha_Bfield;
    else
      sdLumForOuterMini = md.rec[outerMD].dphi * 15.0f / md.rec[outerMD].dz;

    float dAlpha_res_inner = 0.02f / miniDelta * (innerBarrel ? 1.0f : fabs_(zIn) / rtIn);
    float dAlpha_res_outer = 0.02f / miniDelta * (outerBarrel ? 1.0f : fabs_(zOut) / rtOut);
    float dAlpha_res = dAlpha_res_inner + dAlpha_res_outer;

    if (innerBarrel and m.sides[innerLM] == Center)
      thr[0] = dAlpha_Bfield + fsqrt(dAlpha_res * dAlpha_res + sdMuls * sdMuls);
    else
      thr[0] = dAlpha_Bfield +
               fsqrt(dAlpha_res * dAlpha_res + sdMuls * sdMuls + sdLumForInnerMini * sdLumForInnerMini);
    if (outerBarrel and m.sides[outerLM] == Center)
      thr[1] = dAlpha_Bfield + fsqrt(dAlpha_res * dAlpha_res + sdMuls * sdMuls);
    else
      thr[1] = dAlpha_Bfield +
               fsqrt(dAlpha_res * dAlpha_res + sdMuls * sdMuls + sdLumForOuterMini * sdLumForOuterMini);
    thr[2] = dAlpha_Bfield + fsqrt(dAlpha_res * dAlpha_res + sdMuls * sdMuls);
  }

  struct LSValues {
    float dPhi, dPhiMin, dPhiMax, dPhiChange, dPhiChangeMin, dPhiChangeMax;
  };

  // Barrel-barrel segment (SDL/Segment.h:455-565).  dPhiMin/Max and
  // dPhiChangeMin/Max keep their initial value 0.
  LST_HD_BIG bool lsBarrel(const Modules& m,
                       const MiniDoublets& md,
                       uint16_t innerLM,
                       uint16_t outerLM,
                       unsigned int innerMD,
                       unsigned int outerMD,
                       LSValues& v) {
    float sdMuls = (m.subdets[innerLM] == Barrel) ? miniMulsPtScaleBarrel(m.layers[innerLM] - 1) * 3.f / m.ptCut
                                                  : miniMulsPtScaleEndcap(m.layers[innerLM] - 1) * 3.f / m.ptCut;
    const MDRec& rIn = md.rec[innerMD];
    const MDRec& rOut = md.rec[outerMD];
    float xIn = rIn.x, yIn = rIn.y, zIn = rIn.z, rtIn = rIn.rt;
    float xOut = rOut.x, yOut = rOut.y, zOut = rOut.z, rtOut = rOut.rt;

    float sdSlope = rOut.slope;
    float sdPVoff = 0.1f / rtOut;
    float dzDrtScale = rOut.tanSlope / sdSlope;
    const float zGeom = m.layers[innerLM] <= 2 ? 2.f * kPixelPSZpitch : 2.f * kStrip2SZpitch;
    float zLo = zIn + (zIn - kDeltaZLum) * (rtOut / rtIn - 1.f) * (zIn > 0.f ? 1.f : dzDrtScale) - zGeom;
    float zHi = zIn + (zIn + kDeltaZLum) * (rtOut / rtIn - 1.f) * (zIn < 0.f ? 1.f : dzDrtScale) + zGeom;
    if (!((zOut >= zLo) && (zOut <= zHi)))
      return false;

    float sdCut = sdSlope + fsqrt(sdMuls * sdMuls + sdPVoff * sdPVoff);
    v.dPhi = phiMpiPi(rOut.phi - rIn.phi);
    if (!(fabs_(v.dPhi) <= sdCut))
      return false;
    v.dPhiChange = phiMpiPi(phiOf(xOut - xIn, yOut - yIn) - rIn.phi);
    if (!(fabs_(v.dPhiChange) <= sdCut))
      return false;

    float thr[3];
    lsDAlphaThresholds(m, md, xIn, yIn, zIn, rtIn, xOut, yOut, zOut, rtOut, innerLM, outerLM, innerMD, outerMD, thr);
    float innerMDAlpha = rIn.dphichange;
    float outerMDAlpha = rOut.dphichange;
    float dAlphaInnerMDSegment = innerMDAlpha - v.dPhiChange;
    float dAlphaOuterMDSegment = outerMDAlpha - v.dPhiChange;
    float dAlphaInnerMDOuterMD = innerMDAlpha - outerMDAlpha;
    if (!(fabs_(dAlphaInnerMDSegment) < thr[0]))
      return false;
    if (!(fabs_(dAlphaOuterMDSegment) < thr[1]))
      return false;
    return fabs_(dAlphaInnerMDOuterMD) < thr[2];
  }

  // Segment with at least one endcap module (SDL/Segment.h:567-705).
  LST_HD_BIG bool lsEndcap(const Modules& m,
                       const MiniDoublets& md,
                       uint16_t innerLM,
                       uint16_t outerLM,
                       unsigned int innerMD,
                       unsigned int outerMD,
                       LSValues& v) {
    const MDRec& rIn = md.rec[innerMD];
    const MDRec& rOut = md.rec[outerMD];
    float xIn = rIn.x, yIn = rIn.y, zIn = rIn.z, rtIn = rIn.rt;
    float xOut = rOut.x, yOut = rOut.y, zOut = rOut.z, rtOut = rOut.rt;
    bool outerLayerEndcapTwoS = (m.subdets[outerLM] == Endcap) && (m.moduleType[outerLM] == TwoS);
    float sdSlope = rOut.slope;
    float disks2SMinRadius = 60.f;
    float rtGeom = ((rtIn < disks2SMinRadius && rtOut < disks2SMinRadius)
                        ? (2.f * kPixelPSZpitch)
                        : ((rtIn < disks2SMinRadius || rtOut < disks2SMinRadius) ? (kPixelPSZpitch + kStrip2SZpitch)
                                                                                 : (2.f * kStrip2SZpitch)));
    if (!(zIn * zOut >= 0))
      return false;
    float dz = zOut - zIn;
    float dLum = signTransfer(kDeltaZLum, zIn);
    float drtDzScale = sdSlope / rOut.tanSlope;
    float rtLo = fmax_(rtIn * (1.f + dz / (zIn + dLum) * drtDzScale) - rtGeom, rtIn - 0.5f * rtGeom);
    float rtHi = rtIn * (zOut - dLum) / (zIn - dLum) + rtGeom;
    if (!((rtOut >= rtLo) && (rtOut <= rtHi)))
      return false;

    v.dPhi = phiMpiPi(rOut.phi - rIn.phi);
    float sdCut = sdSlope;
    if (outerLayerEndcapTwoS) {
      float dPhiPos_high = phiMpiPi(rOut.highEdgePhi - rIn.phi);
      float dPhiPos_low = phiMpiPi(rOut.lowEdgePhi - rIn.phi);
      v.dPhiMax = fabs_(dPhiPos_high) > fabs_(dPhiPos_low) ? dPhiPos_high : dPhiPos_low;
      v.dPhiMin = fabs_(dPhiPos_high) > fabs_(dPhiPos_low) ? dPhiPos_low : dPhiPos_high;
    } else {
      v.dPhiMax = v.dPhi;
      v.dPhiMin = v.dPhi;
    }
    if (!(fabs_(v.dPhi) <= sdCut))
      return false;

    float dzFrac = dz / zIn;
    v.dPhiChange = v.dPhi / dzFrac * (1.f + dzFrac);
    v.dPhiChangeMin = v.dPhiMin / dzFrac * (1.f + dzFrac);
    v.dPhiChangeMax = v.dPhiMax / dzFrac * (1.f + dzFrac);
    if (!(fabs_(v.dPhiChange) <= sdCut))
      return false;

    float thr[3];
    lsDAlphaThresholds(m, md, xIn, yIn, zIn, rtIn, xOut, yOut, zOut, rtOut, innerLM, outerLM, innerMD, outerMD, thr);
    float innerMDAlpha = rIn.dphichange;
    float outerMDAlpha = rOut.dphichange;
    float dAlphaInnerMDSegment = innerMDAlpha - v.dPhiChange;
    float dAlphaOuterMDSegment = outerMDAlpha - v.dPhiChange;
    float dAlphaInnerMDOuterMD = innerMDAlpha - outerMDAlpha;
    if (!(fabs_(dAlphaInnerMDSegment) < thr[0]))
      return false;
    if (!(fabs_(dAlphaOuterMDSegment) < thr[1]))
      return false;
    return fabs_(dAlphaInnerMDOuterMD) < thr[2];
  }

  LST_HD bool lsSelect(const Modules& m,
                       const MiniDoublets& md,
                       uint16_t innerLM,
                       uint16_t outerLM,
                       unsigned int innerMD,
                       unsigned int outerMD,
                       LSValues& v) {
    v.dPhiMin = 0;
    v.dPhiMax = 0;
    v.dPhiChangeMin = 0;
    v.dPhiChangeMax = 0;
    if (m.subdets[innerLM] == Barrel and m.subdets[outerLM] == Barrel)
      return lsBarrel(m, md, innerLM, outerLM, innerMD, outerMD, v);
    return lsEndcap(m, md, innerLM, outerLM, innerMD, outerMD, v);
  }

  // SDL/Segment.h:358-390
  LST_HD void storeLS(Segments& s,
                      const MiniDoublets& md,
                      unsigned int innerMD,
                      unsigned int outerMD,
                      uint16_t innerLM,
                      uint16_t outerLM,
                      const LSValues& v,
                      unsigned int idx) {
    s.mdIndices[idx * 2] = innerMD;
    s.mdIndices[idx * 2 + 1] = outerMD;
    s.innerLowerModuleIndices[idx] = innerLM;
    s.outerLowerModuleIndices[idx] = outerLM;
    s.innerMiniDoubletAnchorHitIndices[idx] = md.anchorHitIndices[innerMD];
    s.outerMiniDoubletAnchorHitIndices[idx] = md.anchorHitIndices[outerMD];
    s.dPhis[idx] = v.dPhi;
    s.dPhiMins[idx] = v.dPhiMin;
    s.dPhiMaxs[idx] = v.dPhiMax;
    s.dPhiChanges[idx] = v.dPhiChange;
    s.dPhiChangeMins[idx] = v.dPhiChangeMin;
    s.dPhiChangeMaxs[idx] = v.dPhiChangeMax;
  }

  // One pixel line segment: two pixel mini-doublets from the seed's four
  // pseudo-hits, the rz least-squares score and the seed's circle
  // (SDL/Segment.h:1031-1117 with SDL/Segment.h:392-453).
  LST_HD void storePixelSegment(const Modules& m,
                                const Hits& h,
                                MiniDoublets& md,
                                Segments& s,
                                uint16_t pixelModule,
                                unsigned int mdBase,
                                unsigned int lsBase,
                                unsigned int tid,
                                unsigned int hit0,
                                unsigned int hit1,
                                unsigned int hit2,
                                unsigned int hit3,
                                float dPhiChange) {
    unsigned int innerMD = mdBase + 2 * tid;
    unsigned int outerMD = mdBase + 2 * tid + 1;
    unsigned int pls = lsBase + tid;
    MDValues zero{0, 0, 0, 0, 0, 0, 0, 0, 0};
    storeMD(m, h, md, hit0, hit1, pixelModule, zero, innerMD);
    storeMD(m, h, md, hit2, hit3, pixelModule, zero, outerMD);
    // The anchor and outer hits storeMD has just stored (its rule), so that
    // the values below are read from the hits directly rather than back
    // through the stored mini-doublets.
    const bool swap = m.moduleType[pixelModule] == PS and m.moduleLayerType[pixelModule] == Strip;
    const unsigned int inAnchor = swap ? hit1 : hit0, inOuter = swap ? hit0 : hit1;
    const unsigned int outAnchor = swap ? hit3 : hit2, outOuter = swap ? hit2 : hit3;

    float slope = fsinh(h.ys[inOuter]);
    float intercept = h.zs[inAnchor] - slope * h.rts[inAnchor];
    float score_lsq = (h.rts[outAnchor] * slope + intercept) - (h.zs[outAnchor]);
    score_lsq = score_lsq * score_lsq;

    s.mdIndices[pls * 2] = innerMD;
    s.mdIndices[pls * 2 + 1] = outerMD;
    s.innerLowerModuleIndices[pls] = pixelModule;
    s.outerLowerModuleIndices[pls] = pixelModule;
    s.innerMiniDoubletAnchorHitIndices[pls] = hit0;
    s.outerMiniDoubletAnchorHitIndices[pls] = hit2;
    s.dPhiChanges[pls] = dPhiChange;
    s.isDup[tid] = 0;
    s.score[tid] = score_lsq;
    s.pLSHitsIdxs[4 * tid + 0] = h.idxs[inAnchor];
    s.pLSHitsIdxs[4 * tid + 1] = h.idxs[outAnchor];
    s.pLSHitsIdxs[4 * tid + 2] = h.idxs[inOuter];
    s.pLSHitsIdxs[4 * tid + 3] = h.idxs[outOuter];

    float circleRadius = h.xs[inOuter] / (2 * k2Rinv1GeVf);
    float circlePhi = h.zs[inOuter];
    const float inAnchorX = h.xs[inAnchor], inAnchorY = h.ys[inAnchor];
    const float outAnchorX = h.xs[outAnchor], outAnchorY = h.ys[outAnchor];
    float candidateCenterXs[2] = {inAnchorX + circleRadius * fsin(circlePhi), inAnchorX - circleRadius * fsin(circlePhi)};
    float candidateCenterYs[2] = {inAnchorY - circleRadius * fcos(circlePhi), inAnchorY + circleRadius * fcos(circlePhi)};
    float bestChiSquared = kInf;
    int bestIndex = 0;
    for (int i = 0; i < 2; i++) {
      float chiSquared = fabs_(fsqrt((outAnchorX - candidateCenterXs[i]) * (outAnchorX - candidateCenterXs[i]) +
                                     (outAnchorY - candidateCenterYs[i]) * (outAnchorY - candidateCenterYs[i])) -
                               circleRadius);
      if (chiSquared < bestChiSquared) {
        bestChiSquared = chiSquared;
        bestIndex = i;
      }
    }
    s.circleCenterX[tid] = candidateCenterXs[bestIndex];
    s.circleCenterY[tid] = candidateCenterYs[bestIndex];
    s.circleRadius[tid] = circleRadius;
  }

}  // namespace lst
