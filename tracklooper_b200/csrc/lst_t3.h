// Triplet (T3) selection: two line segments sharing a mini-doublet.  Cut
// arithmetic follows SDL/Triplet.h:154-870.
#pragma once

#include "lst_ls.h"

namespace lst {

  // r-z residual of the middle hit against the line through the outer two
  // (SDL/Triplet.h:241-299); layers use the sdlLayers numbering.
  LST_HD bool t3PassRZ(const Modules& m,
                       const MiniDoublets& md,
                       uint16_t lm1,
                       uint16_t lm2,
                       uint16_t lm3,
                       unsigned int md1,
                       unsigned int md2,
                       unsigned int md3) {
    const float r1 = md.rec[md1].rt, r2 = md.rec[md2].rt, r3 = md.rec[md3].rt;
    const float z1 = md.rec[md1].z, z2 = md.rec[md2].z, z3 = md.rec[md3].z;
    const int layer1 = m.sdlLayers[lm1], layer2 = m.sdlLayers[lm2], layer3 = m.sdlLayers[lm3];
    const float residual = z2 - ((z3 - z1) / (r3 - r1) * (r2 - r1) + z1);
    const float ar = fabs_(residual);
    if (layer1 == 12 and layer2 == 13 and layer3 == 14)
      return false;
    if (layer1 == 1 and layer2 == 2 and layer3 == 3)
      return ar < 0.53f;
    if (layer1 == 1 and layer2 == 2 and layer3 == 7)
      return ar < 1;
    if (layer1 == 13 and layer2 == 14 and layer3 == 15)
      return false;
    if (layer1 == 14 and layer2 == 15 and layer3 == 16)
      return false;
    if (layer1 == 1 and layer2 == 7 and layer3 == 8)
      return ar < 1;
    if (layer1 == 2 and layer2 == 3 and layer3 == 4)
      return ar < 1.21f;
    if (layer1 == 2 and layer2 == 3 and layer3 == 7)
      return ar < 1.f;
    if (layer1 == 2 and layer2 == 7 and layer3 == 8)
      return ar < 1.f;
    if (layer1 == 3 and layer2 == 4 and layer3 == 5)
      return ar < 2.7f;
    if (layer1 == 4 and layer2 == 5 and layer3 == 6)
      return ar < 3.06f;
    if (layer1 == 7 and layer2 == 8 and layer3 == 9)
      return ar < 1;
    if (layer1 == 8 and layer2 == 9 and layer3 == 10)
      return ar < 1;
    if (layer1 == 9 and layer2 == 10 and layer3 == 11)
      return ar < 1;
    return ar < 5;
  }

  LST_HD float segmentDr(const MiniDoublets& md, unsigned int a, unsigned int b) {
    return fsqrt((md.rec[b].x - md.rec[a].x) * (md.rec[b].x - md.rec[a].x) +
                 (md.rec[b].y - md.rec[a].y) * (md.rec[b].y - md.rec[a].y));
  }

  // Barrel-barrel-barrel pointing and first beta cut (SDL/Triplet.h:301-402).
  LST_HD_BIG bool t3PointingBBB(const Modules& m,
                            const MiniDoublets& md,
                            const Segments& s,
                            uint16_t lm1,
                            uint16_t lm3,
                            unsigned int md1,
                            unsigned int md2,
                            unsigned int md3,
                            unsigned int innerSeg,
                            float& betaIn) {
    bool isPSIn = (m.moduleType[lm1] == PS);
    bool isPSOut = (m.moduleType[lm3] == PS);
    float rtIn = md.rec[md1].rt, rtMid = md.rec[md2].rt, rtOut = md.rec[md3].rt;
    float zIn = md.rec[md1].z, zMid = md.rec[md2].z, zOut = md.rec[md3].z;
    float alpha1GeVOut = md.rec[md3].slope;
    float rtRatio_OutIn = rtOut / rtIn;
    float dzDrtScale = md.rec[md3].tanSlope / alpha1GeVOut;
    float zpitchIn = (isPSIn ? kPixelPSZpitch : kStrip2SZpitch);
    float zpitchOut = (isPSOut ? kPixelPSZpitch : kStrip2SZpitch);
    const float zHi =
        zIn + (zIn + kDeltaZLum) * (rtRatio_OutIn - 1.f) * (zIn < 0.f ? 1.f : dzDrtScale) + (zpitchIn + zpitchOut);
    const float zLo =
        zIn + (zIn - kDeltaZLum) * (rtRatio_OutIn - 1.f) * (zIn > 0.f ? 1.f : dzDrtScale) - (zpitchIn + zpitchOut);
    if (!((zOut >= zLo) && (zOut <= zHi)))
      return false;

    float drt_OutIn = (rtOut - rtIn);
    float r3In = fsqrt(zIn * zIn + rtIn * rtIn);
    float drt_InSeg = rtMid - rtIn;
    float dz_InSeg = zMid - zIn;
    float dr3_InSeg = fsqrt(rtMid * rtMid + zMid * zMid) - fsqrt(rtIn * rtIn + zIn * zIn);
    float coshEta = dr3_InSeg / drt_InSeg;
    float dzErr = (zpitchIn + zpitchOut) * (zpitchIn + zpitchOut) * 2.f;
    float sdlThetaMulsF = 0.015f * fsqrt(0.1f + 0.2f * (rtOut - rtIn) / 50.f) * fsqrt(r3In / rtIn);
    float sdlMuls = sdlThetaMulsF * 3.f / m.ptCut * 4.f;
    dzErr += sdlMuls * sdlMuls * drt_OutIn * drt_OutIn / 3.f * coshEta * coshEta;
    dzErr = fsqrt(dzErr);
    const float dzMean = dz_InSeg / drt_InSeg * drt_OutIn;
    const float zWindow = dzErr / drt_InSeg * drt_OutIn + (zpitchIn + zpitchOut);
    const float zLoPointed = zIn + dzMean * (zIn > 0.f ? 1.f : dzDrtScale) - zWindow;
    const float zHiPointed = zIn + dzMean * (zIn < 0.f ? 1.f : dzDrtScale) + zWindow;
    bool pass = ((zOut >= zLoPointed) && (zOut <= zHiPointed));

    float alpha_InLo = s.dPhiChanges[innerSeg];
    float tl_axis_x = md.rec[md3].x - md.rec[md1].x;
    float tl_axis_y = md.rec[md3].y - md.rec[md1].y;
    betaIn = alpha_InLo - phiMpiPi(phiOf(tl_axis_x, tl_axis_y) - md.rec[md1].phi);
    float drt_tl_axis = fsqrt(tl_axis_x * tl_axis_x + tl_axis_y * tl_axis_y);
    const float rt_InSeg = segmentDr(md, md1, md2);
    float betaInCut = fasin(fmin_((-rt_InSeg + drt_tl_axis) * k2Rinv1GeVf / m.ptCut, kSinAlphaMax)) + (0.02f / drt_InSeg);
    return pass and (fabs_(betaIn) < betaInCut);
  }

  // Barrel-barrel-endcap / barrel-endcap-endcap (SDL/Triplet.h:404-531).
  LST_HD_BIG bool t3PointingBBE(const Modules& m,
                            const MiniDoublets& md,
                            const Segments& s,
                            uint16_t lm1,
                            uint16_t lm3,
                            unsigned int md1,
                            unsigned int md2,
                            unsigned int md3,
                            unsigned int innerSeg,
                            float& betaIn) {
    bool isPSIn = (m.moduleType[lm1] == PS);
    bool isPSOut = (m.moduleType[lm3] == PS);
    float rtIn = md.rec[md1].rt, rtMid = md.rec[md2].rt, rtOut = md.rec[md3].rt;
    float zIn = md.rec[md1].z, zMid = md.rec[md2].z, zOut = md.rec[md3].z;
    float alpha1GeV_OutLo = md.rec[md3].slope;
    float dzDrtScale = md.rec[md3].tanSlope / alpha1GeV_OutLo;
    float zpitchIn = (isPSIn ? kPixelPSZpitch : kStrip2SZpitch);
    float zpitchOut = (isPSOut ? kPixelPSZpitch : kStrip2SZpitch);
    float zGeom = zpitchIn + zpitchOut;
    if (!(zIn * zOut > 0))
      return false;
    float dLum = signTransfer(kDeltaZLum, zIn);
    bool isOutSgInnerMDPS = m.moduleType[lm3] == PS;
    float rtGeom1 = isOutSgInnerMDPS ? kPixelPSZpitch : kStrip2SZpitch;
    float zGeom1 = signTransfer(zGeom, zIn);
    float rtLo = rtIn * (1.f + (zOut - zIn - zGeom1) / (zIn + zGeom1 + dLum) / dzDrtScale) - rtGeom1;
    float zInForHi = zIn - zGeom1 - dLum;
    if (zInForHi * zIn < 0) {
      zInForHi = signTransfer(0.1f, zIn);
    }
    float rtHi = rtIn * (1.f + (zOut - zIn + zGeom1) / zInForHi) + rtGeom1;
    if (!((rtOut >= rtLo) && (rtOut <= rtHi)))
      return false;

    float rIn = fsqrt(zIn * zIn + rtIn * rtIn);
    const float drtSDIn = rtMid - rtIn;
    const float dzSDIn = zMid - zIn;
    const float dr3SDIn = fsqrt(rtMid * rtMid + zMid * zMid) - fsqrt(rtIn * rtIn + zIn * zIn);
    const float coshEta = dr3SDIn / drtSDIn;
    const float dzOutInAbs = fabs_(zOut - zIn);
    const float multDzDr = dzOutInAbs * coshEta / (coshEta * coshEta - 1.f);
    const float zGeom1_another = kPixelPSZpitch;
    const float kZ = (zOut - zIn) / dzSDIn;
    float drtErr =
        zGeom1_another * zGeom1_another * drtSDIn * drtSDIn / dzSDIn / dzSDIn * (1.f - 2.f * kZ + 2.f * kZ * kZ);
    // The reference evaluates 0.1f + 0.2 * (...) / 50.f in double here.
    const float sdlThetaMulsF =
        0.015f * dsqrt(0.1f + 0.2 * (rtOut - rtIn) / 50.f) * fsqrt(rIn / rtIn);
    const float sdlMuls = sdlThetaMulsF * 3.f / m.ptCut * 4.f;
    drtErr += sdlMuls * sdlMuls * multDzDr * multDzDr / 3.f * coshEta * coshEta;
    drtErr = fsqrt(drtErr);
    bool pass = (kZ >= 0) && (rtOut >= rtLo) && (rtOut <= rtHi);

    float rt_InLo = md.rec[md1].rt;
    float rt_InOut = md.rec[md2].rt;
    float sdIn_alpha = s.dPhiChanges[innerSeg];
    float tl_axis_x = md.rec[md3].x - md.rec[md1].x;
    float tl_axis_y = md.rec[md3].y - md.rec[md1].y;
    betaIn = sdIn_alpha - phiMpiPi(phiOf(tl_axis_x, tl_axis_y) - md.rec[md1].phi);
    float betaInRHmin = betaIn;
    float betaInRHmax = betaIn;
    if (fabs_(betaInRHmin) > fabs_(betaInRHmax)) {
      float swapTemp = betaInRHmin;
      betaInRHmin = betaInRHmax;
      betaInRHmax = swapTemp;
    }
    float sdIn_dr = segmentDr(md, md1, md2);
    float sdIn_d = rt_InOut - rt_InLo;
    float dr = fsqrt(tl_axis_x * tl_axis_x + tl_axis_y * tl_axis_y);
    float betaInCut = fasin(fmin_((-sdIn_dr + dr) * k2Rinv1GeVf / m.ptCut, kSinAlphaMax)) + (0.02f / sdIn_d);
    return pass and (fabs_(betaInRHmin) < betaInCut);
  }

  // Endcap-endcap-endcap (SDL/Triplet.h:533-658).
  LST_HD_BIG bool t3PointingEEE(const Modules& m,
                            const MiniDoublets& md,
                            const Segments& s,
                            uint16_t lm1,
                            uint16_t lm3,
                            unsigned int md1,
                            unsigned int md2,
                            unsigned int md3,
                            unsigned int innerSeg,
                            float& betaIn) {
    float rtIn = md.rec[md1].rt, rtMid = md.rec[md2].rt, rtOut = md.rec[md3].rt;
    float zIn = md.rec[md1].z, zMid = md.rec[md2].z, zOut = md.rec[md3].z;
    float alpha1GeV_Out = md.rec[md3].slope;
    float dzDrtScale = md.rec[md3].tanSlope / alpha1GeV_Out;
    if (!(zIn * zOut > 0))
      return false;
    float dLum = signTransfer(kDeltaZLum, zIn);
    bool isOutSgOuterMDPS = m.moduleType[lm3] == PS;
    bool isInSgInnerMDPS = m.moduleType[lm1] == PS;
    float rtGeom = (isInSgInnerMDPS and isOutSgOuterMDPS)  ? 2.f * kPixelPSZpitch
                   : (isInSgInnerMDPS or isOutSgOuterMDPS) ? kPixelPSZpitch + kStrip2SZpitch
                                                           : 2.f * kStrip2SZpitch;
    float dz = zOut - zIn;
    const float rtLo = rtIn * (1.f + dz / (zIn + dLum) / dzDrtScale) - rtGeom;
    const float rtHi = rtIn * (1.f + dz / (zIn - dLum)) + rtGeom;
    if (!((rtOut >= rtLo) && (rtOut <= rtHi)))
      return false;

    bool isInSgOuterMDPS = m.moduleType[lm3] == PS;
    float drtSDIn = rtMid - rtIn;
    float dzSDIn = zMid - zIn;
    float dr3SDIn = fsqrt(rtMid * rtMid + zMid * zMid) - fsqrt(rtIn * rtIn + zIn * zIn);
    float coshEta = dr3SDIn / drtSDIn;
    float dzOutInAbs = fabs_(zOut - zIn);
    float multDzDr = dzOutInAbs * coshEta / (coshEta * coshEta - 1.f);
    float kZ = (zOut - zIn) / dzSDIn;
    float sdlThetaMulsF = 0.015f * fsqrt(0.1f + 0.2f * (rtOut - rtIn) / 50.f);
    float sdlMuls = sdlThetaMulsF * 3.f / m.ptCut * 4.f;
    float drtErr = fsqrt(kPixelPSZpitch * kPixelPSZpitch * 2.f / (dzSDIn * dzSDIn) * (dzOutInAbs * dzOutInAbs) +
                         sdlMuls * sdlMuls * multDzDr * multDzDr / 3.f * coshEta * coshEta);
    float drtMean = drtSDIn * dzOutInAbs / fabs_(dzSDIn);
    float rtWindow = drtErr + rtGeom;
    float rtLo_point = rtIn + drtMean / dzDrtScale - rtWindow;
    float rtHi_point = rtIn + drtMean + rtWindow;
    bool pass = true;
    if (isInSgInnerMDPS and isInSgOuterMDPS)
      pass = ((kZ >= 0) && (rtOut >= rtLo_point) && (rtOut <= rtHi_point));

    float rt_InLo = md.rec[md1].rt;
    float rt_InOut = md.rec[md2].rt;
    float sdIn_alpha = s.dPhiChanges[innerSeg];
    float tl_axis_x = md.rec[md3].x - md.rec[md1].x;
    float tl_axis_y = md.rec[md3].y - md.rec[md1].y;
    betaIn = sdIn_alpha - phiMpiPi(phiOf(tl_axis_x, tl_axis_y) - md.rec[md1].phi);
    float sdIn_alphaRHmin = s.dPhiChangeMins[innerSeg];
    float sdIn_alphaRHmax = s.dPhiChangeMaxs[innerSeg];
    float betaInRHmin = betaIn + sdIn_alphaRHmin - sdIn_alpha;
    float betaInRHmax = betaIn + sdIn_alphaRHmax - sdIn_alpha;
    if (fabs_(betaInRHmin) > fabs_(betaInRHmax)) {
      float swapTemp = betaInRHmin;
      betaInRHmin = betaInRHmax;
      betaInRHmax = swapTemp;
    }
    float sdIn_dr = segmentDr(md, md1, md2);
    float sdIn_d = rt_InOut - rt_InLo;
    float dr = fsqrt(tl_axis_x * tl_axis_x + tl_axis_y * tl_axis_y);
    float betaInCut = fasin(fmin_((-sdIn_dr + dr) * k2Rinv1GeVf / m.ptCut, kSinAlphaMax)) + (0.02f / sdIn_d);
    return pass and (fabs_(betaInRHmin) < betaInCut);
  }

  // Circle through three points; radius -1 for collinear points
  // (SDL/Triplet.h:762-795).
  LST_HD float circleFrom3(float x1, float y1, float x2, float y2, float x3, float y3, float& g, float& f) {
    float radius = 0.f;
    float denomInv = 1.0f / ((y1 - y3) * (x2 - x3) - (x1 - x3) * (y2 - y3));
    float xy1sqr = x1 * x1 + y1 * y1;
    float xy2sqr = x2 * x2 + y2 * y2;
    float xy3sqr = x3 * x3 + y3 * y3;
    g = 0.5f * ((y3 - y2) * xy1sqr + (y1 - y3) * xy2sqr + (y2 - y1) * xy3sqr) * denomInv;
    f = 0.5f * ((x2 - x3) * xy1sqr + (x3 - x1) * xy2sqr + (x1 - x2) * xy3sqr) * denomInv;
    float c = ((x2 * y3 - x3 * y2) * xy1sqr + (x3 * y1 - x1 * y3) * xy2sqr + (x1 * y2 - x2 * y1) * xy3sqr) * denomInv;
    if (((y1 - y3) * (x2 - x3) - (x1 - x3) * (y2 - y3) == 0) || (g * g + f * f - c < 0))
      radius = -1.f;
    else
      radius = fsqrt(g * g + f * f - c);
    return radius;
  }

  struct T3Values {
    float betaIn, circleRadius, circleCenterX, circleCenterY;
  };

  // SDL/Triplet.h:797-870
  LST_HD bool t3Select(const Modules& m,
                       const MiniDoublets& md,
                       const Segments& s,
                       uint16_t lm1,
                       uint16_t lm2,
                       uint16_t lm3,
                       unsigned int innerSeg,
                       unsigned int outerSeg,
                       T3Values& v) {
    if (s.mdIndices[2 * innerSeg + 1] != s.mdIndices[2 * outerSeg])
      return false;
    unsigned int md1 = s.mdIndices[2 * innerSeg];
    unsigned int md2 = s.mdIndices[2 * outerSeg];
    unsigned int md3 = s.mdIndices[2 * outerSeg + 1];
    if (!t3PassRZ(m, md, lm1, lm2, lm3, md1, md2, md3))
      return false;
    short sub1 = m.subdets[lm1], sub2 = m.subdets[lm2], sub3 = m.subdets[lm3];
    bool pass;
    if (sub1 == Barrel and sub2 == Barrel and sub3 == Barrel)
      pass = t3PointingBBB(m, md, s, lm1, lm3, md1, md2, md3, innerSeg, v.betaIn);
    else if (sub1 == Barrel and sub2 == Barrel and sub3 == Endcap)
      pass = t3PointingBBE(m, md, s, lm1, lm3, md1, md2, md3, innerSeg, v.betaIn);
    else if (sub1 == Barrel and sub2 == Endcap and sub3 == Endcap)
      pass = t3PointingBBE(m, md, s, lm1, lm3, md1, md2, md3, innerSeg, v.betaIn);
    else if (sub1 == Endcap and sub2 == Endcap and sub3 == Endcap)
      pass = t3PointingEEE(m, md, s, lm1, lm3, md1, md2, md3, innerSeg, v.betaIn);
    else
      pass = false;
    if (!pass)
      return false;
    v.circleRadius = circleFrom3(md.rec[md1].x,
                                 md.rec[md1].y,
                                 md.rec[md2].x,
                                 md.rec[md2].y,
                                 md.rec[md3].x,
                                 md.rec[md3].y,
                                 v.circleCenterX,
                                 v.circleCenterY);
    return true;
  }

  // SDL/Triplet.h:181-239
  LST_HD void storeT3(const Modules& m,
                      const MiniDoublets& md,
                      const Segments& s,
                      Triplets& t,
                      unsigned int innerSeg,
                      unsigned int outerSeg,
                      uint16_t lm1,
                      uint16_t lm2,
                      uint16_t lm3,
                      const T3Values& v,
                      unsigned int idx) {
    t.segmentIndices[idx * 2] = innerSeg;
    t.segmentIndices[idx * 2 + 1] = outerSeg;
    t.lowerModuleIndices[idx * 3] = lm1;
    t.lowerModuleIndices[idx * 3 + 1] = lm2;
    t.lowerModuleIndices[idx * 3 + 2] = lm3;
    t.betaIn[idx] = v.betaIn;
    t.circleRadius[idx] = v.circleRadius;
    t.circleCenterX[idx] = v.circleCenterX;
    t.circleCenterY[idx] = v.circleCenterY;
    t.logicalLayers[idx * 3] = m.layers[lm1] + (m.subdets[lm1] == 4) * 6;
    t.logicalLayers[idx * 3 + 1] = m.layers[lm2] + (m.subdets[lm2] == 4) * 6;
    t.logicalLayers[idx * 3 + 2] = m.layers[lm3] + (m.subdets[lm3] == 4) * 6;
    unsigned int md1 = s.mdIndices[2 * innerSeg];
    unsigned int md2 = s.mdIndices[2 * innerSeg + 1];
    unsigned int md3 = s.mdIndices[2 * outerSeg + 1];
    t.hitIndices[idx * 6] = md.anchorHitIndices[md1];
    t.hitIndices[idx * 6 + 1] = md.outerHitIndices[md1];
    t.hitIndices[idx * 6 + 2] = md.anchorHitIndices[md2];
    t.hitIndices[idx * 6 + 3] = md.outerHitIndices[md2];
    t.hitIndices[idx * 6 + 4] = md.anchorHitIndices[md3];
    t.hitIndices[idx * 6 + 5] = md.outerHitIndices[md3];
    // The reference clears these flags for the whole store when it allocates it.
    t.partOfPT5[idx] = 0;
    t.partOfT5[idx] = 0;
    t.partOfPT3[idx] = 0;
  }

}  // namespace lst
