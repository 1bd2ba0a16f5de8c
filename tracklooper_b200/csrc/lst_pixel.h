// Pixel triplets (pT3: pixel line segment + T3) and pixel quintuplets (pT5:
// pixel line segment + T5).  Arithmetic follows SDL/PixelTriplet.h:134-2677.
#pragma once

#include "lst_t5.h"

namespace lst {

  // Layer numbering of the pT3/pT5 chi-squared tables: endcap layers +6, 2S
  // endcap layers another +5 (SDL/PixelTriplet.h:321-335).
  LST_HD int pixelTableLayer(const Modules& m, uint16_t i) {
    return m.layers[i] + 6 * (m.subdets[i] == Endcap) + 5 * (m.subdets[i] == Endcap and m.moduleType[i] == TwoS);
  }

  // Pixel segment against a pair of outer-tracker mini-doublets, barrel outer
  // modules (SDL/PixelTriplet.h:1264-1553).
  LST_HD_BIG bool ptPPBB(const Modules& m,
                     const Ranges& rg,
                     const MiniDoublets& md,
                     const Segments& s,
                     uint16_t pixelModule,
                     uint16_t lmOI,
                     uint16_t lmOO,
                     unsigned int innerSeg,
                     unsigned int outerSeg,
                     unsigned int md1,
                     unsigned int md2,
                     unsigned int md3,
                     unsigned int md4) {
    bool isPS_OutLo = (m.moduleType[lmOI] == PS);
    float rt_InLo = md.anchorPos[md1].rt, rt_InUp = md.anchorPos[md2].rt, rt_OutLo = md.anchorPos[md3].rt, rt_OutUp = md.anchorPos[md4].rt;
    float z_InUp = md.anchorPos[md2].z, z_OutLo = md.anchorPos[md3].z;
    float x_InLo = md.anchorPos[md1].x, x_InUp = md.anchorPos[md2].x, x_OutLo = md.anchorPos[md3].x, x_OutUp = md.anchorPos[md4].x;
    float y_InLo = md.anchorPos[md1].y, y_InUp = md.anchorPos[md2].y, y_OutLo = md.anchorPos[md3].y, y_OutUp = md.anchorPos[md4].y;
    float rt_InOut = rt_InUp;
    // deltaPhi of two anchor hits, from their stored phi (hits.phis is phi()
    // of the same coordinates, so the value is identical)
    if (!(fabs_(phiMpiPi(md.anchorPhi[md3] - md.anchorPhi[md2])) <= 0.5f * float(M_PI)))
      return false;

    unsigned int pls = innerSeg - rg.segmentModuleIndices[pixelModule];
    float ptIn = s.ptIn[pls];
    float px = s.px[pls], py = s.py[pls], pz = s.pz[pls];
    float etaErr = s.etaErr[pls];

    float alpha1GeV_OutLo = md.slope[md3];
    const float rtRatio_OutLoInOut = rt_OutLo / rt_InOut;
    float dzDrtScale = md.tanSlope[md3] / alpha1GeV_OutLo;
    const float zpitch_InLo = 0.05f;
    const float zpitch_InOut = 0.05f;
    float zpitch_OutLo = (isPS_OutLo ? kPixelPSZpitch : kStrip2SZpitch);
    float zGeom = zpitch_InLo + zpitch_OutLo;
    float zHi = z_InUp + (z_InUp + kDeltaZLum) * (rtRatio_OutLoInOut - 1.f) * (z_InUp < 0.f ? 1.f : dzDrtScale) +
                (zpitch_InOut + zpitch_OutLo);
    float zLo = z_InUp + (z_InUp - kDeltaZLum) * (rtRatio_OutLoInOut - 1.f) * (z_InUp > 0.f ? 1.f : dzDrtScale) -
                (zpitch_InOut + zpitch_OutLo);
    if (!((z_OutLo >= zLo) && (z_OutLo <= zHi)))
      return false;

    const float coshEta = fsqrt(ptIn * ptIn + pz * pz) / ptIn;
    const float drt_OutLo_InUp = (rt_OutLo - rt_InUp);
    const float r3_InUp = fsqrt(z_InUp * z_InUp + rt_InUp * rt_InUp);
    float drt_InSeg = rt_InOut - rt_InLo;
    const float sdlThetaMulsF = 0.015f * fsqrt(0.1f + 0.2f * (rt_OutLo - rt_InUp) / 50.f) * fsqrt(r3_InUp / rt_InUp);
    const float sdlMuls = sdlThetaMulsF * 3.f / m.ptCut * 4.f;
    float dzErr = drt_OutLo_InUp * etaErr * coshEta;
    dzErr *= dzErr;
    dzErr += 0.03f * 0.03f;
    dzErr *= 9.f;
    dzErr += sdlMuls * sdlMuls * drt_OutLo_InUp * drt_OutLo_InUp / 3.f * coshEta * coshEta;
    dzErr += zGeom * zGeom;
    dzErr = fsqrt(dzErr);
    const float dzDrIn = pz / ptIn;
    const float zWindow = dzErr / drt_InSeg * drt_OutLo_InUp + zGeom;
    const float dzMean =
        dzDrIn * drt_OutLo_InUp *
        (1.f + drt_OutLo_InUp * drt_OutLo_InUp * 4 * k2Rinv1GeVf * k2Rinv1GeVf / ptIn / ptIn / 24.f);
    float zLoPointed = z_InUp + dzMean - zWindow;
    float zHiPointed = z_InUp + dzMean + zWindow;
    if (!((z_OutLo >= zLoPointed) && (z_OutLo <= zHiPointed)))
      return false;

    const float sdlPVoff = 0.1f / rt_OutLo;
    float sdlCut = alpha1GeV_OutLo + fsqrt(sdlMuls * sdlMuls + sdlPVoff * sdlPVoff);
    float midPointX = 0.5f * (x_InLo + x_OutLo);
    float midPointY = 0.5f * (y_InLo + y_OutLo);
    float diffX = x_OutLo - x_InLo;
    float diffY = y_OutLo - y_InLo;
    float dPhi = deltaPhi(midPointX, midPointY, diffX, diffY);
    if (!(fabs_(dPhi) <= sdlCut))
      return false;

    float alpha_InLo = s.dPhiChanges[innerSeg];
    float alpha_OutLo = s.dPhiChanges[outerSeg];
    bool isEC_lastLayer = m.subdets[lmOO] == Endcap and m.moduleType[lmOO] == TwoS;
    float alpha_OutUp = phiMpiPi(phiOf(x_OutUp - x_OutLo, y_OutUp - y_OutLo) - md.anchorPhi[md4]);
    float tl_axis_x = x_OutUp - x_InUp;
    float tl_axis_y = y_OutUp - y_InUp;
    const float phiTlAxis = phiOf(tl_axis_x, tl_axis_y);
    float betaIn = -phiMpiPi(phiTlAxis - phiOf(px, py));
    float betaInRHmin = betaIn;
    float betaInRHmax = betaIn;
    float betaOut = -alpha_OutUp + phiMpiPi(phiTlAxis - md.anchorPhi[md4]);
    float betaOutRHmin = betaOut;
    float betaOutRHmax = betaOut;
    if (isEC_lastLayer) {
      float hx = md.anchorHighEdgeX[md4], hy = md.anchorHighEdgeY[md4];
      float lx = md.anchorLowEdgeX[md4], ly = md.anchorLowEdgeY[md4];
      float alpha_OutUp_highEdge = deltaPhi(hx, hy, hx - x_OutLo, hy - y_OutLo);
      float alpha_OutUp_lowEdge = deltaPhi(lx, ly, lx - x_OutLo, ly - y_OutLo);
      float tl_axis_highEdge_x = hx - x_InUp;
      float tl_axis_highEdge_y = hy - y_InUp;
      float tl_axis_lowEdge_x = lx - x_InUp;
      float tl_axis_lowEdge_y = ly - y_InUp;
      betaOutRHmin = -alpha_OutUp_highEdge + deltaPhi(hx, hy, tl_axis_highEdge_x, tl_axis_highEdge_y);
      betaOutRHmax = -alpha_OutUp_lowEdge + deltaPhi(lx, ly, tl_axis_lowEdge_x, tl_axis_lowEdge_y);
    }

    float drt_tl_axis = fsqrt(tl_axis_x * tl_axis_x + tl_axis_y * tl_axis_y);
    const float rt_InSeg = fsqrt((x_InUp - x_InLo) * (x_InUp - x_InLo) + (y_InUp - y_InLo) * (y_InUp - y_InLo));
    float betaAv = 0.5f * (betaIn + betaOut);
    float pt_beta = ptIn;
    int lIn = 0;
    int lOut = isEC_lastLayer ? 11 : 5;
    float sdOut_dr = fsqrt((x_OutUp - x_OutLo) * (x_OutUp - x_OutLo) + (y_OutUp - y_OutLo) * (y_OutUp - y_OutLo));
    float sdOut_d = rt_OutUp - rt_OutLo;
    deltaBetaIterations(betaIn, betaOut, betaAv, pt_beta, rt_InSeg, sdOut_dr, drt_tl_axis, lIn);

    const float betaInMMSF =
        (fabs_(betaInRHmin + betaInRHmax) > 0) ? (2.f * betaIn / fabs_(betaInRHmin + betaInRHmax)) : 0.f;
    const float betaOutMMSF =
        (fabs_(betaOutRHmin + betaOutRHmax) > 0) ? (2.f * betaOut / fabs_(betaOutRHmin + betaOutRHmax)) : 0.f;
    betaInRHmin *= betaInMMSF;
    betaInRHmax *= betaInMMSF;
    betaOutRHmin *= betaOutMMSF;
    betaOutRHmax *= betaOutMMSF;

    const float dBetaMuls = sdlThetaMulsF * 4.f / fmin_(fabs_(pt_beta), kPtBetaMax);
    const float alphaInAbsReg = fmax_(fabs_(alpha_InLo), md.slope3[md2]);
    const float alphaOutAbsReg = fmax_(fabs_(alpha_OutLo), md.slope3[md3]);
    const float dBetaInLum = lIn < 11 ? 0.0f : fabs_(alphaInAbsReg * kDeltaZLum / z_InUp);
    const float dBetaOutLum = lOut < 11 ? 0.0f : fabs_(alphaOutAbsReg * kDeltaZLum / z_OutLo);
    const float dBetaLum2 = (dBetaInLum + dBetaOutLum) * (dBetaInLum + dBetaOutLum);
    const float sinDPhi = fsin(dPhi);
    const float dBetaRIn2 = 0;
    float dBetaROut = 0;
    if (isEC_lastLayer) {
      dBetaROut = (fsqrt(md.anchorHighEdgeX[md4] * md.anchorHighEdgeX[md4] + md.anchorHighEdgeY[md4] * md.anchorHighEdgeY[md4]) -
                   fsqrt(md.anchorLowEdgeX[md4] * md.anchorLowEdgeX[md4] + md.anchorLowEdgeY[md4] * md.anchorLowEdgeY[md4])) *
                  sinDPhi / drt_tl_axis;
    }
    const float dBetaROut2 = dBetaROut * dBetaROut;
    float betaOutCut = fasin(fmin_(drt_tl_axis * k2Rinv1GeVf / m.ptCut, kSinAlphaMax)) + (0.02f / sdOut_d) +
                       fsqrt(dBetaLum2 + dBetaMuls * dBetaMuls);
    if (!(fabs_(betaOut) < betaOutCut))
      return false;
    const float dBetaRes = 0.02f / fmin_(sdOut_d, drt_InSeg);
    return betaDifferenceCut(betaIn, betaOut, betaInRHmin, betaInRHmax, betaOutRHmin, betaOutRHmax, dBetaRes, dBetaMuls,
                             dBetaLum2, dBetaRIn2, dBetaROut2);
  }

  // Pixel segment against an endcap pair (SDL/PixelTriplet.h:1555-1862).
  LST_HD_BIG bool ptPPEE(const Modules& m,
                     const Ranges& rg,
                     const MiniDoublets& md,
                     const Segments& s,
                     uint16_t pixelModule,
                     uint16_t lmOI,
                     uint16_t lmOO,
                     unsigned int innerSeg,
                     unsigned int outerSeg,
                     unsigned int md1,
                     unsigned int md2,
                     unsigned int md3,
                     unsigned int md4) {
    bool isPS_OutLo = (m.moduleType[lmOI] == PS);
    float z_InUp = md.anchorPos[md2].z;
    float z_OutLo = md.anchorPos[md3].z;
    if (!(z_InUp * z_OutLo > 0))
      return false;
    float rt_InLo = md.anchorPos[md1].rt, rt_InUp = md.anchorPos[md2].rt, rt_OutLo = md.anchorPos[md3].rt, rt_OutUp = md.anchorPos[md4].rt;
    float x_InLo = md.anchorPos[md1].x, x_InUp = md.anchorPos[md2].x, x_OutLo = md.anchorPos[md3].x, x_OutUp = md.anchorPos[md4].x;
    float y_InLo = md.anchorPos[md1].y, y_InUp = md.anchorPos[md2].y, y_OutLo = md.anchorPos[md3].y, y_OutUp = md.anchorPos[md4].y;
    unsigned int pls = innerSeg - rg.segmentModuleIndices[pixelModule];
    float ptIn = s.ptIn[pls];
    float px = s.px[pls], py = s.py[pls], pz = s.pz[pls];
    float etaErr = s.etaErr[pls];

    const float zpitch_InLo = 0.05f;
    float zpitch_OutLo = (isPS_OutLo ? kPixelPSZpitch : kStrip2SZpitch);
    float zGeom = zpitch_InLo + zpitch_OutLo;
    const float sdlSlope = md.slope[md3];
    const float dzDrtScale = md.tanSlope[md3] / sdlSlope;
    const float dLum = signTransfer(kDeltaZLum, z_InUp);
    bool isOutSgInnerMDPS = m.moduleType[lmOI] == PS;
    const float rtGeom1 = isOutSgInnerMDPS ? kPixelPSZpitch : kStrip2SZpitch;
    const float zGeom1 = signTransfer(zGeom, z_InUp);
    float rtLo = rt_InUp * (1.f + (z_OutLo - z_InUp - zGeom1) / (z_InUp + zGeom1 + dLum) / dzDrtScale) - rtGeom1;
    float zInForHi = z_InUp - zGeom1 - dLum;
    if (zInForHi * z_InUp < 0)
      zInForHi = signTransfer(0.1f, z_InUp);
    float rtHi = rt_InUp * (1.f + (z_OutLo - z_InUp + zGeom1) / zInForHi) + rtGeom1;
    if (!((rt_OutLo >= rtLo) && (rt_OutLo <= rtHi)))
      return false;

    const float dzOutInAbs = fabs_(z_OutLo - z_InUp);
    const float coshEta = fsqrt(ptIn * ptIn + pz * pz) / ptIn;
    const float multDzDr = dzOutInAbs * coshEta / (coshEta * coshEta - 1.f);
    const float r3_InUp = fsqrt(z_InUp * z_InUp + rt_InUp * rt_InUp);
    const float sdlThetaMulsF = 0.015f * fsqrt(0.1f + 0.2f * (rt_OutLo - rt_InUp) / 50.f) * fsqrt(r3_InUp / rt_InUp);
    const float sdlMuls = sdlThetaMulsF * 3.f / m.ptCut * 4.f;
    float drtErr = etaErr * multDzDr;
    drtErr *= drtErr;
    drtErr += 0.03f * 0.03f;
    drtErr *= 9.f;
    drtErr += sdlMuls * sdlMuls * multDzDr * multDzDr / 3.f * coshEta * coshEta;
    drtErr = fsqrt(drtErr);
    const float drtDzIn = fabs_(ptIn / pz);
    const float drt_OutLo_InUp = (rt_OutLo - rt_InUp);
    const float rtWindow = drtErr + rtGeom1;
    const float drtMean =
        drtDzIn * dzOutInAbs *
        (1.f - drt_OutLo_InUp * drt_OutLo_InUp * 4 * k2Rinv1GeVf * k2Rinv1GeVf / ptIn / ptIn / 24.f);
    const float rtLo_point = rt_InUp + drtMean - rtWindow;
    const float rtHi_point = rt_InUp + drtMean + rtWindow;
    if (!((rt_OutLo >= rtLo_point) && (rt_OutLo <= rtHi_point)))
      return false;

    const float alpha1GeV_OutLo = md.slope[md3];
    const float sdlPVoff = 0.1f / rt_OutLo;
    float sdlCut = alpha1GeV_OutLo + fsqrt(sdlMuls * sdlMuls + sdlPVoff * sdlPVoff);
    float midPointX = 0.5f * (x_InLo + x_OutLo);
    float midPointY = 0.5f * (y_InLo + y_OutLo);
    float diffX = x_OutLo - x_InLo;
    float diffY = y_OutLo - y_InLo;
    float dPhi = deltaPhi(midPointX, midPointY, diffX, diffY);
    if (!(fabs_(dPhi) <= sdlCut))
      return false;

    float alpha_InLo = s.dPhiChanges[innerSeg];
    float alpha_OutLo = s.dPhiChanges[outerSeg];
    bool isEC_lastLayer = m.subdets[lmOO] == Endcap and m.moduleType[lmOO] == TwoS;
    float alpha_OutUp = phiMpiPi(phiOf(x_OutUp - x_OutLo, y_OutUp - y_OutLo) - md.anchorPhi[md4]);
    float tl_axis_x = x_OutUp - x_InUp;
    float tl_axis_y = y_OutUp - y_InUp;
    const float phiTlAxis = phiOf(tl_axis_x, tl_axis_y);
    float betaIn = -phiMpiPi(phiTlAxis - phiOf(px, py));
    float betaInRHmin = betaIn;
    float betaInRHmax = betaIn;
    float betaOut = -alpha_OutUp + phiMpiPi(phiTlAxis - md.anchorPhi[md4]);
    float betaOutRHmin = betaOut;
    float betaOutRHmax = betaOut;
    if (isEC_lastLayer) {
      float hx = md.anchorHighEdgeX[md4], hy = md.anchorHighEdgeY[md4];
      float lx = md.anchorLowEdgeX[md4], ly = md.anchorLowEdgeY[md4];
      float alpha_OutUp_highEdge = deltaPhi(hx, hy, hx - x_OutLo, hy - y_OutLo);
      float alpha_OutUp_lowEdge = deltaPhi(lx, ly, lx - x_OutLo, ly - y_OutLo);
      float tl_axis_highEdge_x = hx - x_InUp;
      float tl_axis_highEdge_y = hy - y_InUp;
      float tl_axis_lowEdge_x = lx - x_InUp;
      float tl_axis_lowEdge_y = ly - y_InUp;
      betaOutRHmin = -alpha_OutUp_highEdge + deltaPhi(hx, hy, tl_axis_highEdge_x, tl_axis_highEdge_y);
      betaOutRHmax = -alpha_OutUp_lowEdge + deltaPhi(lx, ly, tl_axis_lowEdge_x, tl_axis_lowEdge_y);
    }

    float drt_tl_axis = fsqrt(tl_axis_x * tl_axis_x + tl_axis_y * tl_axis_y);
    const float rt_InSeg = fsqrt((x_InUp - x_InLo) * (x_InUp - x_InLo) + (y_InUp - y_InLo) * (y_InUp - y_InLo));
    float betaAv = 0.5f * (betaIn + betaOut);
    float pt_beta = ptIn;
    int lIn = 0;
    int lOut = isEC_lastLayer ? 11 : 5;
    float sdOut_dr = fsqrt((x_OutUp - x_OutLo) * (x_OutUp - x_OutLo) + (y_OutUp - y_OutLo) * (y_OutUp - y_OutLo));
    float sdOut_d = rt_OutUp - rt_OutLo;
    deltaBetaIterations(betaIn, betaOut, betaAv, pt_beta, rt_InSeg, sdOut_dr, drt_tl_axis, lIn);

    const float betaInMMSF =
        (fabs_(betaInRHmin + betaInRHmax) > 0) ? (2.f * betaIn / fabs_(betaInRHmin + betaInRHmax)) : 0.f;
    const float betaOutMMSF =
        (fabs_(betaOutRHmin + betaOutRHmax) > 0) ? (2.f * betaOut / fabs_(betaOutRHmin + betaOutRHmax)) : 0.f;
    betaInRHmin *= betaInMMSF;
    betaInRHmax *= betaInMMSF;
    betaOutRHmin *= betaOutMMSF;
    betaOutRHmax *= betaOutMMSF;

    const float dBetaMuls = sdlThetaMulsF * 4.f / fmin_(fabs_(pt_beta), kPtBetaMax);
    const float alphaInAbsReg = fmax_(fabs_(alpha_InLo), md.slope3[md2]);
    const float alphaOutAbsReg = fmax_(fabs_(alpha_OutLo), md.slope3[md3]);
    const float dBetaInLum = lIn < 11 ? 0.0f : fabs_(alphaInAbsReg * kDeltaZLum / z_InUp);
    const float dBetaOutLum = lOut < 11 ? 0.0f : fabs_(alphaOutAbsReg * kDeltaZLum / z_OutLo);
    const float dBetaLum2 = (dBetaInLum + dBetaOutLum) * (dBetaInLum + dBetaOutLum);
    const float sinDPhi = fsin(dPhi);
    const float dBetaRIn2 = 0;
    float dBetaROut = 0;
    if (isEC_lastLayer) {
      dBetaROut = (fsqrt(md.anchorHighEdgeX[md4] * md.anchorHighEdgeX[md4] + md.anchorHighEdgeY[md4] * md.anchorHighEdgeY[md4]) -
                   fsqrt(md.anchorLowEdgeX[md4] * md.anchorLowEdgeX[md4] + md.anchorLowEdgeY[md4] * md.anchorLowEdgeY[md4])) *
                  sinDPhi / drt_tl_axis;
    }
    const float dBetaROut2 = dBetaROut * dBetaROut;
    float betaOutCut = fasin(fmin_(drt_tl_axis * k2Rinv1GeVf / m.ptCut, kSinAlphaMax)) + (0.02f / sdOut_d) +
                       fsqrt(dBetaLum2 + dBetaMuls * dBetaMuls);
    if (!(fabs_(betaOut) < betaOutCut))
      return false;
    float drt_InSeg = rt_InUp - rt_InLo;
    const float dBetaRes = 0.02f / fmin_(sdOut_d, drt_InSeg);
    return betaDifferenceCut(betaIn, betaOut, betaInRHmin, betaInRHmax, betaOutRHmin, betaOutRHmax, dBetaRes, dBetaMuls,
                             dBetaLum2, dBetaRIn2, dBetaROut2);
  }

  // Dispatch (SDL/PixelTriplet.h:206-314).
  LST_HD bool ptPixelTracklet(const Modules& m,
                              const Ranges& rg,
                              const MiniDoublets& md,
                              const Segments& s,
                              uint16_t pixelModule,
                              uint16_t lmOI,
                              uint16_t lmOO,
                              unsigned int innerSeg,
                              unsigned int outerSeg) {
    short sOI = m.subdets[lmOI], sOO = m.subdets[lmOO];
    unsigned int md1 = s.mdIndices[2 * innerSeg], md2 = s.mdIndices[2 * innerSeg + 1];
    unsigned int md3 = s.mdIndices[2 * outerSeg], md4 = s.mdIndices[2 * outerSeg + 1];
    if (sOI == Barrel and (sOO == Barrel or sOO == Endcap))
      return ptPPBB(m, rg, md, s, pixelModule, lmOI, lmOO, innerSeg, outerSeg, md1, md2, md3, md4);
    if (sOI == Endcap and sOO == Endcap)
      return ptPPEE(m, rg, md, s, pixelModule, lmOI, lmOO, innerSeg, outerSeg, md1, md2, md3, md4);
    return false;
  }

  // ------------------------------------------------------------- pT3 cuts
  LST_HD bool pt3PassRZ(const Modules& m, uint16_t a, uint16_t b, uint16_t c, float rz) {
    const int layer1 = pixelTableLayer(m, a), layer2 = pixelTableLayer(m, b), layer3 = pixelTableLayer(m, c);
    if (layer1 == 8 and layer2 == 9 and layer3 == 10)
      return rz < 13.6067f;
    if (layer1 == 8 and layer2 == 9 and layer3 == 15)
      return rz < 5.5953f;
    if (layer1 == 7 and layer2 == 8 and layer3 == 9)
      return rz < 3.9263f;
    if (layer1 == 1 and layer2 == 2 and layer3 == 3)
      return rz < 9.4377f;
    if (layer1 == 1 and layer2 == 2 and layer3 == 7)
      return rz < 9.9975f;
    if (layer1 == 1 and layer2 == 7 and layer3 == 8)
      return rz < 8.6369f;
    if (layer1 == 2 and layer2 == 3 and layer3 == 7)
      return rz < 37.945f;
    if (layer1 == 2 and layer2 == 3 and layer3 == 12)
      return rz < 43.0167f;
    if (layer1 == 2 and layer2 == 3 and layer3 == 4)
      return rz < 8.6923f;
    if (layer1 == 2 and layer2 == 7 and layer3 == 8)
      return rz < 11.9672f;
    if (layer1 == 2 and layer2 == 7 and layer3 == 13)
      return rz < 16.2133f;
    return true;
  }

  LST_HD bool pt3PassRPhi(const Modules& m, uint16_t a, uint16_t b, uint16_t c, float chi) {
    const int layer1 = pixelTableLayer(m, a), layer2 = pixelTableLayer(m, b), layer3 = pixelTableLayer(m, c);
    if (layer1 == 8 and layer2 == 9 and layer3 == 10)
      return chi < 7.003f;
    if (layer1 == 8 and layer2 == 9 and layer3 == 15)
      return chi < 0.5f;
    if (layer1 == 7 and layer2 == 8 and layer3 == 9)
      return chi < 8.046f;
    if (layer1 == 7 and layer2 == 8 and layer3 == 14)
      return chi < 0.575f;
    if (layer1 == 1 and layer2 == 2 and layer3 == 7)
      return chi < 5.304f;
    if (layer1 == 1 and layer2 == 2 and layer3 == 3)
      return chi < 10.6211f;
    if (layer1 == 1 and layer2 == 7 and layer3 == 8)
      return chi < 4.617f;
    if (layer1 == 2 and layer2 == 7 and layer3 == 8)
      return chi < 8.046f;
    if (layer1 == 2 and layer2 == 7 and layer3 == 13)
      return chi < 0.435f;
    if (layer1 == 2 and layer2 == 3 and layer3 == 7)
      return chi < 9.244f;
    if (layer1 == 2 and layer2 == 3 and layer3 == 12)
      return chi < 0.287f;
    if (layer1 == 2 and layer2 == 3 and layer3 == 4)
      return chi < 18.509f;
    return true;
  }

  LST_HD bool pt3PassRPhiInwards(const Modules& m, uint16_t a, uint16_t b, uint16_t c, float chi) {
    const int layer1 = pixelTableLayer(m, a), layer2 = pixelTableLayer(m, b), layer3 = pixelTableLayer(m, c);
    if (layer1 == 7 and layer2 == 8 and layer3 == 9)
      return chi < 22016.8055f;
    if (layer1 == 7 and layer2 == 8 and layer3 == 14)
      return chi < 935179.56807f;
    if (layer1 == 8 and layer2 == 9 and layer3 == 10)
      return chi < 29064.12959f;
    if (layer1 == 8 and layer2 == 9 and layer3 == 15)
      return chi < 935179.5681f;
    if (layer1 == 1 and layer2 == 2 and layer3 == 3)
      return chi < 1370.0113195101474f;
    if (layer1 == 1 and layer2 == 2 and layer3 == 7)
      return chi < 5492.110048314815f;
    if (layer1 == 2 and layer2 == 3 and layer3 == 4)
      return chi < 4160.410806470067f;
    if (layer1 == 1 and layer2 == 7 and layer3 == 8)
      return chi < 29064.129591225726f;
    if (layer1 == 2 and layer2 == 3 and layer3 == 7)
      return chi < 12634.215376250893f;
    if (layer1 == 2 and layer2 == 3 and layer3 == 12)
      return chi < 353821.69361145404f;
    if (layer1 == 2 and layer2 == 7 and layer3 == 8)
      return chi < 33393.26076341235f;
    if (layer1 == 2 and layer2 == 7 and layer3 == 13)
      return chi < 935179.5680742573f;
    return true;
  }

  // Inverse-radius compatibility of the pixel segment and the triplet
  // (SDL/PixelTriplet.h:616-735).  kind: 0 BBB, 1 BBE, 2 BEE, 3 EEE.
  LST_HD bool pt3RadiusCriterion(int kind, float pixelRadius, float pixelRadiusError, float tripletRadius) {
    const bool highPt = pixelRadius > 2.0f * kR1GeVf;
    float tE, pE;
    switch (kind) {
      case 0:
        tE = highPt ? 0.6588f : 0.15624f;
        pE = highPt ? 0.6375f : 0.17235f;
        break;
      case 1:
        tE = highPt ? 0.8557f : 0.45972f;
        pE = highPt ? 0.6805f : 0.19644f;
        break;
      case 2:
        tE = highPt ? 2.3548f : 1.59294f;
        pE = highPt ? 2.2091f : 0.255181f;
        break;
      default:
        tE = highPt ? 2.436f : 1.7006f;
        pE = highPt ? 2.286f : 0.26367f;
        break;
    }
    float tripletRadiusInvMax = (1 + tE) / tripletRadius;
    float tripletRadiusInvMin = fmax_((1 - tE) / tripletRadius, 0.0f);
    float pixelRadiusInvMax = fmax_((1 + pE) / pixelRadius, 1.f / (pixelRadius - pixelRadiusError));
    float pixelRadiusInvMin = fmin_((1 - pE) / pixelRadius, 1.f / (pixelRadius + pixelRadiusError));
    if (kind >= 2)
      pixelRadiusInvMin = fmax_(pixelRadiusInvMin, 0.0f);
    return intervalsOverlap(tripletRadiusInvMin, tripletRadiusInvMax, pixelRadiusInvMin, pixelRadiusInvMax);
  }

  // Helix r-z residuals of the triplet hits from the pixel state
  // (SDL/PixelTriplet.h:736-823).
  LST_HD_BIG float pt3RZChi2(const Modules& m,
                         const uint16_t* lm,
                         const float* rtPix,
                         const float* xPix,
                         const float* yPix,
                         const float* zPix,
                         const float* rts,
                         const float* zs,
                         float pixelSegmentPx,
                         float pixelSegmentPy,
                         float pixelSegmentPz,
                         int pixelSegmentCharge) {
    float residual = 0;
    float error = 0;
    float RMSE = 0;
    float Px = pixelSegmentPx, Py = pixelSegmentPy, Pz = pixelSegmentPz;
    int charge = pixelSegmentCharge;
    float x1 = xPix[1] / 100;
    float y1 = yPix[1] / 100;
    float z1 = zPix[1] / 100;
    float r1 = rtPix[1] / 100;
    float Bz = kMagneticField;
    float a = -0.299792 * Bz * charge;
    for (int i = 0; i < 3; i++) {
      float zsi = zs[i] / 100;
      float rtsi = rts[i] / 100;
      uint16_t lmi = lm[i];
      const int moduleType = m.moduleType[lmi];
      const int moduleSide = m.sides[lmi];
      const int moduleSubdet = m.subdets[lmi];
      float diffr = 0, diffz = 0;
      float p = fsqrt(Px * Px + Py * Py + Pz * Pz);
      float rou = a / p;
      if (moduleSubdet == Endcap) {
        float s = (zsi - z1) * p / Pz;
        float x = x1 + Px / a * fsin(rou * s) - Py / a * (1 - fcos(rou * s));
        float y = y1 + Py / a * fsin(rou * s) + Px / a * (1 - fcos(rou * s));
        diffr = fabs_(rtsi - fsqrt(x * x + y * y)) * 100;
      }
      if (moduleSubdet == Barrel) {
        float paraA = r1 * r1 + 2 * (Px * Px + Py * Py) / (a * a) + 2 * (y1 * Px - x1 * Py) / a - rtsi * rtsi;
        float paraB = 2 * (x1 * Px + y1 * Py) / a;
        float paraC = 2 * (y1 * Px - x1 * Py) / a + 2 * (Px * Px + Py * Py) / (a * a);
        float A = paraB * paraB + paraC * paraC;
        float B = 2 * paraA * paraB;
        float C = paraA * paraA - paraC * paraC;
        float sol1 = (-B + fsqrt(B * B - 4 * A * C)) / (2 * A);
        float sol2 = (-B - fsqrt(B * B - 4 * A * C)) / (2 * A);
        float solz1 = fasin(sol1) / rou * Pz / p + z1;
        float solz2 = fasin(sol2) / rou * Pz / p + z1;
        float diffz1 = fabs_(solz1 - zsi) * 100;
        float diffz2 = fabs_(solz2 - zsi) * 100;
        diffz = fmin_(diffz1, diffz2);
      }
      residual = moduleSubdet == Barrel ? diffz : diffr;
      if (moduleType == 0)
        error = 0.15f;
      else
        error = 5.0f;
      if (moduleType == 0 and moduleSubdet == Barrel and moduleSide != Center) {
        float drdz = m.drdzs[lmi];
        error /= fsqrt(1 + drdz * drdz);
      }
      RMSE += (residual * residual) / (error * error);
    }
    RMSE = fsqrt(0.2f * RMSE);
    return RMSE;
  }

  LST_HD float pixelInwardsChi2(float g, float f, float r, const float* xPix, const float* yPix) {
    float residual = (xPix[0] - g) * (xPix[0] - g) + (yPix[0] - f) * (yPix[0] - f) - r * r;
    float chiSquared = residual * residual;
    residual = (xPix[1] - g) * (xPix[1] - g) + (yPix[1] - f) * (yPix[1] - f) - r * r;
    chiSquared += residual * residual;
    chiSquared *= 0.5f;
    return chiSquared;
  }

  struct PT3Values {
    float pixelRadius, pixelRadiusError, tripletRadius, centerX, centerY, rzChiSquared, rPhiChiSquared,
        rPhiChiSquaredInwards;
  };

  // The opening test of pt3Select below, alone: the radius criterion of the
  // pLS and triplet radii (the cheapest test, and the first one evaluated).
  LST_HD bool pt3RadiusPass(const Modules& m, const Ranges& rg, const Segments& s, const Triplets& t,
                            unsigned int plsIndex, unsigned int t3) {
    uint16_t pixelModule = s.innerLowerModuleIndices[plsIndex];
    uint16_t lmL = t.lowerModuleIndices[3 * t3], lmM = t.lowerModuleIndices[3 * t3 + 1],
             lmU = t.lowerModuleIndices[3 * t3 + 2];
    unsigned int pls = plsIndex - rg.segmentModuleIndices[pixelModule];
    const float pixelRadius = s.ptIn[pls] * kR1GeVf;
    const float pixelRadiusError = s.ptErr[pls] * kR1GeVf;
    int kind = (m.subdets[lmL] == Endcap) ? 3 : (m.subdets[lmM] == Endcap) ? 2 : (m.subdets[lmU] == Endcap) ? 1 : 0;
    return pt3RadiusCriterion(kind, pixelRadius, pixelRadiusError, t.circleRadius[t3]);
  }

  // The second test of pt3Select below, alone: the pixel tracklet algorithm
  // of the pLS with the triplet's inner segment.
  LST_HD bool pt3FirstTracklet(const Modules& m, const Ranges& rg, const MiniDoublets& md, const Segments& s,
                               const Triplets& t, unsigned int plsIndex, unsigned int t3) {
    const uint16_t pixelModule = s.innerLowerModuleIndices[plsIndex];
    return ptPixelTracklet(m, rg, md, s, pixelModule, t.lowerModuleIndices[3 * t3], t.lowerModuleIndices[3 * t3 + 1],
                           plsIndex, t.segmentIndices[2 * t3]);
  }

  // pLS x T3 selection (SDL/PixelTriplet.h:826-1023).
  LST_HD bool pt3Select(const Modules& m,
                        const Ranges& rg,
                        const MiniDoublets& md,
                        const Segments& s,
                        const Triplets& t,
                        unsigned int plsIndex,
                        unsigned int t3,
                        bool runChiSquaredCuts,
                        PT3Values& v) {
    uint16_t pixelModule = s.innerLowerModuleIndices[plsIndex];
    uint16_t lmL = t.lowerModuleIndices[3 * t3], lmM = t.lowerModuleIndices[3 * t3 + 1],
             lmU = t.lowerModuleIndices[3 * t3 + 2];
    unsigned int pls = plsIndex - rg.segmentModuleIndices[pixelModule];
    float pixelSegmentPt = s.ptIn[pls];
    float pixelSegmentPtError = s.ptErr[pls];
    v.pixelRadius = pixelSegmentPt * kR1GeVf;
    v.pixelRadiusError = pixelSegmentPtError * kR1GeVf;
    v.tripletRadius = t.circleRadius[t3];
    // The radius criterion is the reference's third test; every test here is
    // a pure function of the pair, so testing this cheap one first changes no
    // outcome and skips the two tracklet algorithms for most pairs.
    int kind = (m.subdets[lmL] == Endcap) ? 3 : (m.subdets[lmM] == Endcap) ? 2 : (m.subdets[lmU] == Endcap) ? 1 : 0;
    if (!pt3RadiusCriterion(kind, v.pixelRadius, v.pixelRadiusError, v.tripletRadius))
      return false;
    if (!ptPixelTracklet(m, rg, md, s, pixelModule, lmL, lmM, plsIndex, t.segmentIndices[2 * t3]))
      return false;
    if (!ptPixelTracklet(m, rg, md, s, pixelModule, lmM, lmU, plsIndex, t.segmentIndices[2 * t3 + 1]))
      return false;

    float pixelG = s.circleCenterX[pls];
    float pixelF = s.circleCenterY[pls];
    float pixelRadiusPCA = s.circleRadius[pls];
    unsigned int pixelInnerMD = s.mdIndices[2 * plsIndex];
    unsigned int pixelOuterMD = s.mdIndices[2 * plsIndex + 1];
    unsigned int innerSeg = t.segmentIndices[2 * t3], outerSeg = t.segmentIndices[2 * t3 + 1];
    unsigned int md1 = s.mdIndices[2 * innerSeg], md2 = s.mdIndices[2 * innerSeg + 1], md3 = s.mdIndices[2 * outerSeg + 1];
    float xs[3] = {md.anchorPos[md1].x, md.anchorPos[md2].x, md.anchorPos[md3].x};
    float ys[3] = {md.anchorPos[md1].y, md.anchorPos[md2].y, md.anchorPos[md3].y};
    float g = t.circleCenterX[t3];
    float f = t.circleCenterY[t3];

    uint16_t lm3[3] = {lmL, lmM, lmU};
    if (runChiSquaredCuts and pixelSegmentPt < 5.0f) {
      float rts[3] = {md.anchorPos[md1].rt, md.anchorPos[md2].rt, md.anchorPos[md3].rt};
      float zs[3] = {md.anchorPos[md1].z, md.anchorPos[md2].z, md.anchorPos[md3].z};
      float rtPix[2] = {md.anchorPos[pixelInnerMD].rt, md.anchorPos[pixelOuterMD].rt};
      float xPix[2] = {md.anchorPos[pixelInnerMD].x, md.anchorPos[pixelOuterMD].x};
      float yPix[2] = {md.anchorPos[pixelInnerMD].y, md.anchorPos[pixelOuterMD].y};
      float zPix[2] = {md.anchorPos[pixelInnerMD].z, md.anchorPos[pixelOuterMD].z};
      v.rzChiSquared = pt3RZChi2(m, lm3, rtPix, xPix, yPix, zPix, rts, zs, s.px[pls], s.py[pls], s.pz[pls], s.charge[pls]);
      if (!pt3PassRZ(m, lmL, lmM, lmU, v.rzChiSquared))
        return false;
    } else {
      v.rzChiSquared = -1;
    }

    float delta1[3], delta2[3], slopes[3];
    bool isFlat[3];
    regressionSigmas(m, lm3, delta1, delta2, slopes, isFlat, 3, true);
    v.rPhiChiSquared = circleChi2(3, xs, ys, delta1, delta2, slopes, isFlat, pixelG, pixelF, pixelRadiusPCA);
    if (runChiSquaredCuts and pixelSegmentPt < 5.0f) {
      if (!pt3PassRPhi(m, lmL, lmM, lmU, v.rPhiChiSquared))
        return false;
    }
    float xPix[2] = {md.anchorPos[pixelInnerMD].x, md.anchorPos[pixelOuterMD].x};
    float yPix[2] = {md.anchorPos[pixelInnerMD].y, md.anchorPos[pixelOuterMD].y};
    v.rPhiChiSquaredInwards = pixelInwardsChi2(g, f, v.tripletRadius, xPix, yPix);
    if (runChiSquaredCuts and pixelSegmentPt < 5.0f) {
      if (!pt3PassRPhiInwards(m, lmL, lmM, lmU, v.rPhiChiSquaredInwards))
        return false;
    }
    v.centerX = 0;
    v.centerY = 0;
    return true;
  }

  // SDL/PixelTriplet.h:134-204 with the eta/phi/pt/score of :1117-1124.
  LST_HD void storePT3(const Modules& m,
                       const MiniDoublets& md,
                       const Segments& s,
                       const Triplets& t,
                       PixelTriplets& p,
                       unsigned int plsIndex,
                       unsigned int pls,
                       unsigned int t3,
                       short layer2_adjustment,
                       const PT3Values& v,
                       unsigned int idx) {
    unsigned int etaMD = s.mdIndices[2 * t.segmentIndices[2 * t3] + layer2_adjustment];
    p.pixelSegmentIndices[idx] = plsIndex;
    p.tripletIndices[idx] = t3;
    p.pixelRadius[idx] = v.pixelRadius;
    p.tripletRadius[idx] = v.tripletRadius;
    p.pt[idx] = s.ptIn[pls];
    p.eta[idx] = md.anchorEta[etaMD];
    p.phi[idx] = md.anchorPhi[etaMD];
    p.eta_pix[idx] = s.eta[pls];
    p.phi_pix[idx] = s.phi[pls];
    p.isDup[idx] = 0;
    p.partOfPT5[idx] = 0;
    p.score[idx] = v.rPhiChiSquared + v.rPhiChiSquaredInwards;
    p.centerX[idx] = v.centerX;
    p.centerY[idx] = v.centerY;
    p.logicalLayers[5 * idx] = 0;
    p.logicalLayers[5 * idx + 1] = 0;
    p.logicalLayers[5 * idx + 2] = t.logicalLayers[t3 * 3];
    p.logicalLayers[5 * idx + 3] = t.logicalLayers[t3 * 3 + 1];
    p.logicalLayers[5 * idx + 4] = t.logicalLayers[t3 * 3 + 2];
    p.lowerModuleIndices[5 * idx] = s.innerLowerModuleIndices[plsIndex];
    p.lowerModuleIndices[5 * idx + 1] = s.outerLowerModuleIndices[plsIndex];
    p.lowerModuleIndices[5 * idx + 2] = t.lowerModuleIndices[3 * t3];
    p.lowerModuleIndices[5 * idx + 3] = t.lowerModuleIndices[3 * t3 + 1];
    p.lowerModuleIndices[5 * idx + 4] = t.lowerModuleIndices[3 * t3 + 2];
    unsigned int pixelInnerMD = s.mdIndices[2 * plsIndex];
    unsigned int pixelOuterMD = s.mdIndices[2 * plsIndex + 1];
    p.hitIndices[10 * idx] = md.anchorHitIndices[pixelInnerMD];
    p.hitIndices[10 * idx + 1] = md.outerHitIndices[pixelInnerMD];
    p.hitIndices[10 * idx + 2] = md.anchorHitIndices[pixelOuterMD];
    p.hitIndices[10 * idx + 3] = md.outerHitIndices[pixelOuterMD];
    for (int i = 0; i < 6; ++i)
      p.hitIndices[10 * idx + 4 + i] = t.hitIndices[6 * t3 + i];
    p.pixelRadiusError[idx] = v.pixelRadiusError;
    p.rPhiChiSquared[idx] = v.rPhiChiSquared;
    p.rPhiChiSquaredInwards[idx] = v.rPhiChiSquaredInwards;
    p.rzChiSquared[idx] = v.rzChiSquared;
  }

  // ------------------------------------------------------------- pT5 cuts
  LST_HD bool pt5PassRZ(const Modules& m, const uint16_t* lm, float rz) {
    const int layer1 = pixelTableLayer(m, lm[0]), layer2 = pixelTableLayer(m, lm[1]), layer3 = pixelTableLayer(m, lm[2]),
              layer4 = pixelTableLayer(m, lm[3]), layer5 = pixelTableLayer(m, lm[4]);
    if (layer1 == 1 and layer2 == 2 and layer3 == 3) {
      if (layer4 == 12 and layer5 == 13)
        return rz < 451.141f;
      else if (layer4 == 4 and layer5 == 12)
        return rz < 392.654f;
      else if (layer4 == 4 and layer5 == 5)
        return rz < 225.322f;
      else if (layer4 == 7 and layer5 == 13)
        return rz < 595.546f;
      else if (layer4 == 7 and layer5 == 8)
        return rz < 196.111f;
    } else if (layer1 == 1 and layer2 == 2 and layer3 == 7) {
      if (layer4 == 13 and layer5 == 14)
        return rz < 297.446f;
      else if (layer4 == 8 and layer5 == 14)
        return rz < 451.141f;
      else if (layer4 == 8 and layer5 == 9)
        return rz < 518.339f;
    } else if (layer1 == 1 and layer2 == 7 and layer3 == 8) {
      if (layer4 == 9 and layer5 == 10)
        return rz < 341.75f;
      else if (layer4 == 9 and layer5 == 15)
        return rz < 341.75f;
    } else if (layer1 == 2 and layer2 == 3 and layer3 == 4) {
      if (layer4 == 12 and layer5 == 13)
        return rz < 392.655f;
      else if (layer4 == 5 and layer5 == 12)
        return rz < 341.75f;
      else if (layer4 == 5 and layer5 == 6)
        return rz < 112.537f;
    } else if (layer1 == 2 and layer2 == 3 and layer4 == 7) {
      // As in the reference, this branch tests layer4 == 7 and then requires
      // layer4 to be 13 or 8, so it never cuts.
      if (layer4 == 13 and layer5 == 14)
        return rz < 595.545f;
      else if (layer4 == 8 and layer5 == 14)
        return rz < 74.198f;
    } else if (layer1 == 2 and layer2 == 7 and layer3 == 8) {
      if (layer4 == 14 and layer5 == 15)
        return rz < 518.339f;
      else if (layer4 == 9 and layer5 == 10)
        return rz < 8.046f;
      else if (layer4 == 9 and layer5 == 15)
        return rz < 451.141f;
    } else if (layer1 == 3 and layer2 == 7 and layer3 == 8 and layer4 == 14 and layer5 == 15) {
      return rz < 56.207f;
    } else if (layer1 == 7 and layer2 == 8 and layer3 == 9) {
      if (layer4 == 10 and layer5 == 11)
        return rz < 64.578f;
      else if (layer4 == 10 and layer5 == 16)
        return rz < 85.250f;
      else if (layer4 == 15 and layer5 == 16)
        return rz < 85.250f;
    }
    return true;
  }

  LST_HD bool pt5PassRPhi(const Modules& m, const uint16_t* lm, float chi) {
    const int layer1 = pixelTableLayer(m, lm[0]), layer2 = pixelTableLayer(m, lm[1]), layer3 = pixelTableLayer(m, lm[2]),
              layer4 = pixelTableLayer(m, lm[3]), layer5 = pixelTableLayer(m, lm[4]);
    if (layer1 == 1 and layer2 == 2 and layer3 == 3) {
      if (layer4 == 12 and layer5 == 13)
        return chi < 48.921f;
      else if (layer4 == 4 and layer5 == 12)
        return chi < 97.948f;
      else if (layer4 == 4 and layer5 == 5)
        return chi < 129.3f;
      else if (layer4 == 7 and layer5 == 13)
        return chi < 56.21f;
      else if (layer4 == 7 and layer5 == 8)
        return chi < 74.198f;
    } else if (layer1 == 1 and layer2 == 2 and layer3 == 7) {
      if (layer4 == 13 and layer5 == 14)
        return chi < 21.265f;
      else if (layer4 == 8 and layer5 == 14)
        return chi < 37.058f;
      else if (layer4 == 8 and layer5 == 9)
        return chi < 42.578f;
    } else if (layer1 == 1 and layer2 == 7 and layer3 == 8) {
      if (layer4 == 9 and layer5 == 10)
        return chi < 32.253f;
      else if (layer4 == 9 and layer5 == 15)
        return chi < 37.058f;
    } else if (layer1 == 2 and layer2 == 3 and layer3 == 4) {
      if (layer4 == 12 and layer5 == 13)
        return chi < 97.947f;
      else if (layer4 == 5 and layer5 == 12)
        return chi < 129.3f;
      else if (layer4 == 5 and layer5 == 6)
        return chi < 170.68f;
    } else if (layer1 == 2 and layer2 == 3 and layer3 == 7) {
      if (layer4 == 13 and layer5 == 14)
        return chi < 48.92f;
      else if (layer4 == 8 and layer5 == 14)
        return chi < 74.2f;
    } else if (layer1 == 2 and layer2 == 7 and layer3 == 8) {
      if (layer4 == 14 and layer5 == 15)
        return chi < 42.58f;
      else if (layer4 == 9 and layer5 == 10)
        return chi < 37.06f;
      else if (layer4 == 9 and layer5 == 15)
        return chi < 48.92f;
    } else if (layer1 == 3 and layer2 == 7 and layer3 == 8 and layer4 == 14 and layer5 == 15) {
      return chi < 85.25f;
    } else if (layer1 == 7 and layer2 == 8 and layer3 == 9) {
      if (layer4 == 10 and layer5 == 11)
        return chi < 42.58f;
      else if (layer4 == 10 and layer5 == 16)
        return chi < 37.06f;
      else if (layer4 == 15 and layer5 == 16)
        return chi < 37.06f;
    }
    return true;
  }

  LST_HD bool pt5PassRPhiInwards(const Modules& m, const uint16_t* lm, float chi) {
    const int layer1 = pixelTableLayer(m, lm[0]), layer2 = pixelTableLayer(m, lm[1]), layer3 = pixelTableLayer(m, lm[2]),
              layer4 = pixelTableLayer(m, lm[3]), layer5 = pixelTableLayer(m, lm[4]);
    if (layer1 == 1 and layer2 == 2 and layer3 == 3) {
      if (layer4 == 12 and layer5 == 13)
        return chi < 451.141f;
      else if (layer4 == 4 and layer5 == 12)
        return chi < 786.173f;
      else if (layer4 == 4 and layer5 == 5)
        return chi < 595.545f;
      else if (layer4 == 7 and layer5 == 13)
        return chi < 581.339f;
      else if (layer4 == 7 and layer5 == 8)
        return chi < 112.537f;
    } else if (layer1 == 1 and layer2 == 2 and layer3 == 7) {
      if (layer4 == 13 and layer5 == 14)
        return chi < 225.322f;
      else if (layer4 == 8 and layer5 == 14)
        return chi < 1192.402f;
      else if (layer4 == 8 and layer5 == 9)
        return chi < 786.173f;
    } else if (layer1 == 1 and layer2 == 7 and layer3 == 8) {
      if (layer4 == 9 and layer5 == 10)
        return chi < 1037.817f;
      else if (layer4 == 9 and layer5 == 15)
        return chi < 1808.536f;
    } else if (layer1 == 2 and layer2 == 3 and layer3 == 4) {
      if (layer4 == 12 and layer5 == 13)
        return chi < 684.253f;
      else if (layer4 == 5 and layer5 == 12)
        return chi < 684.253f;
      else if (layer4 == 5 and layer5 == 6)
        return chi < 684.253f;
    } else if (layer1 == 2 and layer2 == 3 and layer3 == 7) {
      if (layer4 == 13 and layer5 == 14)
        return chi < 451.141f;
      else if (layer4 == 8 and layer5 == 14)
        return chi < 518.34f;
    } else if (layer1 == 2 and layer2 == 7 and layer3 == 8) {
      if (layer4 == 14 and layer5 == 15)
        return chi < 2077.92f;
      else if (layer4 == 9 and layer5 == 10)
        return chi < 74.20f;
      else if (layer4 == 9 and layer5 == 15)
        return chi < 1808.536f;
    } else if (layer1 == 3 and layer2 == 7 and layer3 == 8 and layer4 == 14 and layer5 == 15) {
      return chi < 786.173f;
    } else if (layer1 == 7 and layer2 == 8 and layer3 == 9) {
      if (layer4 == 10 and layer5 == 11)
        return chi < 1574.076f;
      else if (layer4 == 10 and layer5 == 16)
        return chi < 5492.11f;
      else if (layer4 == 15 and layer5 == 16)
        return chi < 2743.037f;
    }
    return true;
  }

  // Straight-line r-z residuals from the two pixel anchors (SDL/PixelTriplet.h:2636-2677).
  LST_HD_BIG float pt5RZChi2(const Modules& m, const uint16_t* lm, const float* rtPix, const float* zPix, const float* rts,
                         const float* zs) {
    float slope = (zPix[1] - zPix[0]) / (rtPix[1] - rtPix[0]);
    float residual = 0;
    float error = 0;
    float RMSE = 0;
    for (int i = 0; i < 5; i++) {
      uint16_t lmi = lm[i];
      const int moduleType = m.moduleType[lmi];
      const int moduleSide = m.sides[lmi];
      const int moduleSubdet = m.subdets[lmi];
      residual = (moduleSubdet == Barrel) ? (zs[i] - zPix[0]) - slope * (rts[i] - rtPix[0])
                                          : (rts[i] - rtPix[0]) - (zs[i] - zPix[0]) / slope;
      const float drdz = m.drdzs[lmi];
      if (moduleType == 0)
        error = 0.15f;
      else
        error = 5.0f;
      if (moduleType == 0 and moduleSubdet == Barrel and moduleSide != Center)
        error /= fsqrt(1.f + drdz * drdz);
      RMSE += (residual * residual) / (error * error);
    }
    RMSE = fsqrt(0.2f * RMSE);
    return RMSE;
  }

  struct PT5Values {
    float rzChiSquared, rPhiChiSquared, rPhiChiSquaredInwards, pixelRadius, quintupletRadius, centerX, centerY;
  };

  // pLS x T5 selection (SDL/PixelTriplet.h:2480-2634).
  LST_HD bool pt5Select(const Modules& m,
                        const Ranges& rg,
                        const MiniDoublets& md,
                        const Segments& s,
                        const Triplets& t,
                        const Quintuplets& q,
                        unsigned int plsIndex,
                        unsigned int t5,
                        unsigned int pls,
                        PT5Values& v) {
    unsigned int innerT3 = q.tripletIndices[2 * t5];
    unsigned int outerT3 = q.tripletIndices[2 * t5 + 1];
    PT3Values tmp;
    if (!pt3Select(m, rg, md, s, t, plsIndex, innerT3, false, tmp))
      return false;
    unsigned int seg1 = t.segmentIndices[2 * innerT3], seg2 = t.segmentIndices[2 * innerT3 + 1];
    unsigned int seg3 = t.segmentIndices[2 * outerT3], seg4 = t.segmentIndices[2 * outerT3 + 1];
    unsigned int pixelInnerMD = s.mdIndices[2 * plsIndex];
    unsigned int pixelOuterMD = s.mdIndices[2 * plsIndex + 1];
    unsigned int mdi[5] = {
        s.mdIndices[2 * seg1], s.mdIndices[2 * seg2], s.mdIndices[2 * seg2 + 1], s.mdIndices[2 * seg3 + 1], s.mdIndices[2 * seg4 + 1]};
    uint16_t lm[5];
    for (int i = 0; i < 5; ++i)
      lm[i] = q.lowerModuleIndices[5 * t5 + i];
    float zPix[2] = {md.anchorPos[pixelInnerMD].z, md.anchorPos[pixelOuterMD].z};
    float rtPix[2] = {md.anchorPos[pixelInnerMD].rt, md.anchorPos[pixelOuterMD].rt};
    float zs[5], rts[5], xs[5], ys[5];
    for (int i = 0; i < 5; ++i) {
      zs[i] = md.anchorPos[mdi[i]].z;
      rts[i] = md.anchorPos[mdi[i]].rt;
      xs[i] = md.anchorPos[mdi[i]].x;
      ys[i] = md.anchorPos[mdi[i]].y;
    }
    v.rzChiSquared = 0;
    v.centerX = s.circleCenterX[pls];
    v.centerY = s.circleCenterY[pls];
    v.pixelRadius = s.circleRadius[pls];
    if (v.pixelRadius < 5.0f * kR1GeVf) {
      v.rzChiSquared = pt5RZChi2(m, lm, rtPix, zPix, rts, zs);
      if (!pt5PassRZ(m, lm, v.rzChiSquared))
        return false;
    }
    float T5CenterX = q.regressionG[t5];
    float T5CenterY = q.regressionF[t5];
    v.quintupletRadius = q.regressionRadius[t5];
    float delta1[5], delta2[5], slopes[5];
    bool isFlat[5];
    regressionSigmas(m, lm, delta1, delta2, slopes, isFlat, 5, true);
    v.rPhiChiSquared = circleChi2(5, xs, ys, delta1, delta2, slopes, isFlat, v.centerX, v.centerY, v.pixelRadius);
    if (v.pixelRadius < 5.0f * kR1GeVf) {
      if (!pt5PassRPhi(m, lm, v.rPhiChiSquared))
        return false;
    }
    float xPix[2] = {md.anchorPos[pixelInnerMD].x, md.anchorPos[pixelOuterMD].x};
    float yPix[2] = {md.anchorPos[pixelInnerMD].y, md.anchorPos[pixelOuterMD].y};
    v.rPhiChiSquaredInwards = pixelInwardsChi2(T5CenterX, T5CenterY, v.quintupletRadius, xPix, yPix);
    if (q.regressionRadius[t5] < 5.0f * kR1GeVf) {
      if (!pt5PassRPhiInwards(m, lm, v.rPhiChiSquaredInwards))
        return false;
    }
    v.centerX = (v.centerX + T5CenterX) / 2;
    v.centerY = (v.centerY + T5CenterY) / 2;
    return true;
  }

  // SDL/PixelTriplet.h:1961-2036 and the flags set at :2778-2781.
  LST_HD void storePT5(const MiniDoublets& md,
                       Segments& s,
                       Triplets& t,
                       Quintuplets& q,
                       PixelQuintuplets& p,
                       unsigned int plsIndex,
                       unsigned int pls,
                       unsigned int t5,
                       const PT5Values& v,
                       unsigned int idx) {
    p.pixelIndices[idx] = plsIndex;
    p.T5Indices[idx] = t5;
    p.isDup[idx] = 0;
    p.score[idx] = v.rPhiChiSquared;
    p.eta[idx] = q.eta[t5];
    p.phi[idx] = q.phi[t5];
    p.pixelRadius[idx] = v.pixelRadius;
    p.quintupletRadius[idx] = v.quintupletRadius;
    p.centerX[idx] = v.centerX;
    p.centerY[idx] = v.centerY;
    p.logicalLayers[7 * idx] = 0;
    p.logicalLayers[7 * idx + 1] = 0;
    for (int i = 0; i < 5; ++i)
      p.logicalLayers[7 * idx + 2 + i] = q.logicalLayers[t5 * 5 + i];
    p.lowerModuleIndices[7 * idx] = s.innerLowerModuleIndices[plsIndex];
    p.lowerModuleIndices[7 * idx + 1] = s.outerLowerModuleIndices[plsIndex];
    for (int i = 0; i < 5; ++i)
      p.lowerModuleIndices[7 * idx + 2 + i] = q.lowerModuleIndices[t5 * 5 + i];
    unsigned int pixelInnerMD = s.mdIndices[2 * plsIndex];
    unsigned int pixelOuterMD = s.mdIndices[2 * plsIndex + 1];
    p.hitIndices[14 * idx] = md.anchorHitIndices[pixelInnerMD];
    p.hitIndices[14 * idx + 1] = md.outerHitIndices[pixelInnerMD];
    p.hitIndices[14 * idx + 2] = md.anchorHitIndices[pixelOuterMD];
    p.hitIndices[14 * idx + 3] = md.outerHitIndices[pixelOuterMD];
    for (int i = 0; i < 10; ++i)
      p.hitIndices[14 * idx + 4 + i] = q.hitIndices[10 * t5 + i];
    p.rzChiSquared[idx] = v.rzChiSquared;
    p.rPhiChiSquared[idx] = v.rPhiChiSquared;
    p.rPhiChiSquaredInwards[idx] = v.rPhiChiSquaredInwards;
    t.partOfPT5[q.tripletIndices[2 * t5]] = 1;
    t.partOfPT5[q.tripletIndices[2 * t5 + 1]] = 1;
    s.partOfPT5[pls] = 1;
    q.partOfPT5[t5] = 1;
  }

}  // namespace lst
