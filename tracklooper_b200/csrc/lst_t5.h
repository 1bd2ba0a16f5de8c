// Quintuplet (T5) selection: two triplets sharing a mini-doublet, with
// T4-style beta cuts, radius matching, r-z chi-squared, a weighted circle fit
// and either the T5 DNN or an r-phi chi-squared cut.  Arithmetic follows
// SDL/Quintuplet.h:142-2984 and SDL/NeuralNetwork.h:21-165.
#pragma once

#include "lst_t3.h"

namespace lst {

  // Weights of the T5 classifier: 38 -> 32 (ReLU) -> 32 (ReLU) -> 1 (sigmoid),
  // stored transposed as in SDL/NeuralNetworkWeights.h (w0[in][out]).
  struct T5DnnWeights {
    float w0[38 * 32];
    float b0[32];
    float w2[32 * 32];
    float b2[32];
    float w4[32];
    float b4[1];
  };
  constexpr int kT5DnnParams = 38 * 32 + 32 + 32 * 32 + 32 + 32 + 1;

  LST_HD bool intervalsOverlap(float firstMin, float firstMax, float secondMin, float secondMax) {
    return ((firstMin <= secondMin) && (secondMin < firstMax)) || ((secondMin < firstMin) && (firstMin < secondMax));
  }

  // ---------------------------------------------------------- beta updates
  // SDL/Quintuplet.h:1370-1465 (identical in SDL/PixelTriplet.h:1167-1262).
  LST_HD void deltaBetaIterations(
      float& betaIn, float& betaOut, float& betaAv, float& pt_beta, float sdIn_dr, float sdOut_dr, float dr, float lIn) {
    if (lIn == 0) {
      betaOut += signTransfer(fasin(fmin_(sdOut_dr * k2Rinv1GeVf / fabs_(pt_beta), kSinAlphaMax)), betaOut);
      return;
    }
    if (betaIn * betaOut > 0.f and
        (fabs_(pt_beta) < 4.f * kPtBetaMax or (lIn >= 11 and fabs_(pt_beta) < 8.f * kPtBetaMax))) {
      const float betaInUpd = betaIn + signTransfer(fasin(fmin_(sdIn_dr * k2Rinv1GeVf / fabs_(pt_beta), kSinAlphaMax)), betaIn);
      const float betaOutUpd =
          betaOut + signTransfer(fasin(fmin_(sdOut_dr * k2Rinv1GeVf / fabs_(pt_beta), kSinAlphaMax)), betaOut);
      betaAv = 0.5f * (betaInUpd + betaOutUpd);
      const float pt_beta_inv = 1.f / fabs_(dr * k2Rinv1GeVf / fsin(betaAv));
      betaIn += signTransfer(fasin(fmin_(sdIn_dr * k2Rinv1GeVf * pt_beta_inv, kSinAlphaMax)), betaIn);
      betaOut += signTransfer(fasin(fmin_(sdOut_dr * k2Rinv1GeVf * pt_beta_inv, kSinAlphaMax)), betaOut);
      betaAv = 0.5f * (betaIn + betaOut);
      pt_beta = dr * k2Rinv1GeVf / fsin(betaAv);
    } else if (lIn < 11 && fabs_(betaOut) < 0.2f * fabs_(betaIn) && fabs_(pt_beta) < 12.f * kPtBetaMax) {
      const float pt_betaIn = dr * k2Rinv1GeVf / fsin(betaIn);
      const float betaInUpd = betaIn + signTransfer(fasin(fmin_(sdIn_dr * k2Rinv1GeVf / fabs_(pt_betaIn), kSinAlphaMax)), betaIn);
      const float betaOutUpd =
          betaOut + signTransfer(fasin(fmin_(sdOut_dr * k2Rinv1GeVf / fabs_(pt_betaIn), kSinAlphaMax)), betaIn);
      betaAv = (fabs_(betaOut) > 0.2f * fabs_(betaIn)) ? (0.5f * (betaInUpd + betaOutUpd)) : betaInUpd;
      pt_beta = dr * k2Rinv1GeVf / fsin(betaAv);
      betaIn += signTransfer(fasin(fmin_(sdIn_dr * k2Rinv1GeVf / fabs_(pt_beta), kSinAlphaMax)), betaIn);
      betaOut += signTransfer(fasin(fmin_(sdOut_dr * k2Rinv1GeVf / fabs_(pt_beta), kSinAlphaMax)), betaIn);
      betaAv = 0.5f * (betaIn + betaOut);
      pt_beta = dr * k2Rinv1GeVf / fsin(betaAv);
    }
  }

  // Final beta-difference cut shared by the T4-style algorithms.
  LST_HD bool betaDifferenceCut(float betaIn,
                                float betaOut,
                                float betaInRHmin,
                                float betaInRHmax,
                                float betaOutRHmin,
                                float betaOutRHmax,
                                float dBetaRes,
                                float dBetaMuls,
                                float dBetaLum2,
                                float dBetaRIn2,
                                float dBetaROut2) {
    float dBetaCut2 = (dBetaRes * dBetaRes * 2.0f + dBetaMuls * dBetaMuls + dBetaLum2 + dBetaRIn2 + dBetaROut2 +
                       0.25f * (fabs_(betaInRHmin - betaInRHmax) + fabs_(betaOutRHmin - betaOutRHmax)) *
                           (fabs_(betaInRHmin - betaInRHmax) + fabs_(betaOutRHmin - betaOutRHmax)));
    float dBeta = betaIn - betaOut;
    return dBeta * dBeta <= dBetaCut2;
  }

  // Indices of the four modules / mini-doublets seen by a T4-style check.
  struct T4Input {
    uint16_t lmII, lmIO, lmOI, lmOO;  // inner-inner, inner-outer, outer-inner, outer-outer modules
    unsigned int innerSeg, outerSeg;
    unsigned int md1, md2, md3, md4;
  };

  // Barrel-barrel-barrel-(barrel|endcap) (SDL/Quintuplet.h:1467-1746).
  LST_HD_BIG bool t4BBBB(const Modules& m, const MiniDoublets& md, const Segments& s, const T4Input& q) {
    bool isPS_InLo = (m.moduleType[q.lmII] == PS);
    bool isPS_OutLo = (m.moduleType[q.lmOI] == PS);
    float rt_InLo = md.anchorPos[q.md1].rt, rt_InOut = md.anchorPos[q.md2].rt, rt_OutLo = md.anchorPos[q.md3].rt;
    float z_InLo = md.anchorPos[q.md1].z, z_InOut = md.anchorPos[q.md2].z, z_OutLo = md.anchorPos[q.md3].z;
    float alpha1GeV_OutLo = md.slope[q.md3];
    float rtRatio_OutLoInLo = rt_OutLo / rt_InLo;
    float dzDrtScale = md.tanSlope[q.md3] / alpha1GeV_OutLo;
    float zpitch_InLo = (isPS_InLo ? kPixelPSZpitch : kStrip2SZpitch);
    float zpitch_OutLo = (isPS_OutLo ? kPixelPSZpitch : kStrip2SZpitch);
    float zHi = z_InLo + (z_InLo + kDeltaZLum) * (rtRatio_OutLoInLo - 1.f) * (z_InLo < 0.f ? 1.f : dzDrtScale) +
                (zpitch_InLo + zpitch_OutLo);
    float zLo = z_InLo + (z_InLo - kDeltaZLum) * (rtRatio_OutLoInLo - 1.f) * (z_InLo > 0.f ? 1.f : dzDrtScale) -
                (zpitch_InLo + zpitch_OutLo);
    if (!((z_OutLo >= zLo) && (z_OutLo <= zHi)))
      return false;

    float drt_OutLo_InLo = (rt_OutLo - rt_InLo);
    float r3_InLo = fsqrt(z_InLo * z_InLo + rt_InLo * rt_InLo);
    float drt_InSeg = rt_InOut - rt_InLo;
    float dz_InSeg = z_InOut - z_InLo;
    float dr3_InSeg = fsqrt(rt_InOut * rt_InOut + z_InOut * z_InOut) - fsqrt(rt_InLo * rt_InLo + z_InLo * z_InLo);
    float coshEta = dr3_InSeg / drt_InSeg;
    float dzErr = (zpitch_InLo + zpitch_OutLo) * (zpitch_InLo + zpitch_OutLo) * 2.f;
    float sdlThetaMulsF = 0.015f * fsqrt(0.1f + 0.2f * (rt_OutLo - rt_InLo) / 50.f) * fsqrt(r3_InLo / rt_InLo);
    float sdlMuls = sdlThetaMulsF * 3.f / m.ptCut * 4.f;
    dzErr += sdlMuls * sdlMuls * drt_OutLo_InLo * drt_OutLo_InLo / 3.f * coshEta * coshEta;
    dzErr = fsqrt(dzErr);
    const float dzMean = dz_InSeg / drt_InSeg * drt_OutLo_InLo;
    const float zWindow = dzErr / drt_InSeg * drt_OutLo_InLo + (zpitch_InLo + zpitch_OutLo);
    float zLoPointed = z_InLo + dzMean * (z_InLo > 0.f ? 1.f : dzDrtScale) - zWindow;
    float zHiPointed = z_InLo + dzMean * (z_InLo < 0.f ? 1.f : dzDrtScale) + zWindow;
    if (!((z_OutLo >= zLoPointed) && (z_OutLo <= zHiPointed)))
      return false;

    float sdlPVoff = 0.1f / rt_OutLo;
    float sdlCut = alpha1GeV_OutLo + fsqrt(sdlMuls * sdlMuls + sdlPVoff * sdlPVoff);
    float deltaPhiPos = phiMpiPi(md.anchorPhi[q.md4] - md.anchorPhi[q.md2]);
    if (!(fabs_(deltaPhiPos) <= sdlCut))
      return false;
    float midPointX = 0.5f * (md.anchorPos[q.md1].x + md.anchorPos[q.md3].x);
    float midPointY = 0.5f * (md.anchorPos[q.md1].y + md.anchorPos[q.md3].y);
    float diffX = md.anchorPos[q.md3].x - md.anchorPos[q.md1].x;
    float diffY = md.anchorPos[q.md3].y - md.anchorPos[q.md1].y;
    float dPhi = deltaPhi(midPointX, midPointY, diffX, diffY);
    if (!(fabs_(dPhi) <= sdlCut))
      return false;

    float alpha_InLo = s.dPhiChanges[q.innerSeg];
    float alpha_OutLo = s.dPhiChanges[q.outerSeg];
    bool isEC_lastLayer = m.subdets[q.lmOO] == Endcap and m.moduleType[q.lmOO] == TwoS;
    float alpha_OutUp = phiMpiPi(phiOf(md.anchorPos[q.md4].x - md.anchorPos[q.md3].x, md.anchorPos[q.md4].y - md.anchorPos[q.md3].y) -
                                 md.anchorPhi[q.md4]);
    float tl_axis_x = md.anchorPos[q.md4].x - md.anchorPos[q.md1].x;
    float tl_axis_y = md.anchorPos[q.md4].y - md.anchorPos[q.md1].y;
    float betaIn = alpha_InLo - phiMpiPi(phiOf(tl_axis_x, tl_axis_y) - md.anchorPhi[q.md1]);
    float betaInRHmin = betaIn;
    float betaInRHmax = betaIn;
    float betaOut = -alpha_OutUp + phiMpiPi(phiOf(tl_axis_x, tl_axis_y) - md.anchorPhi[q.md4]);
    float betaOutRHmin = betaOut;
    float betaOutRHmax = betaOut;
    if (isEC_lastLayer) {
      float alpha_OutUp_highEdge =
          phiMpiPi(phiOf(md.anchorHighEdgeX[q.md4] - md.anchorPos[q.md3].x, md.anchorHighEdgeY[q.md4] - md.anchorPos[q.md3].y) -
                   md.anchorHighEdgePhi[q.md4]);
      float alpha_OutUp_lowEdge =
          phiMpiPi(phiOf(md.anchorLowEdgeX[q.md4] - md.anchorPos[q.md3].x, md.anchorLowEdgeY[q.md4] - md.anchorPos[q.md3].y) -
                   md.anchorLowEdgePhi[q.md4]);
      float tl_axis_highEdge_x = md.anchorHighEdgeX[q.md4] - md.anchorPos[q.md1].x;
      float tl_axis_highEdge_y = md.anchorHighEdgeY[q.md4] - md.anchorPos[q.md1].y;
      float tl_axis_lowEdge_x = md.anchorLowEdgeX[q.md4] - md.anchorPos[q.md1].x;
      float tl_axis_lowEdge_y = md.anchorLowEdgeY[q.md4] - md.anchorPos[q.md1].y;
      betaOutRHmin = -alpha_OutUp_highEdge +
                     phiMpiPi(phiOf(tl_axis_highEdge_x, tl_axis_highEdge_y) - md.anchorHighEdgePhi[q.md4]);
      betaOutRHmax =
          -alpha_OutUp_lowEdge + phiMpiPi(phiOf(tl_axis_lowEdge_x, tl_axis_lowEdge_y) - md.anchorLowEdgePhi[q.md4]);
    }

    float drt_tl_axis = fsqrt(tl_axis_x * tl_axis_x + tl_axis_y * tl_axis_y);
    float corrF = 1.f;
    const float rt_InSeg = segmentDr(md, q.md1, q.md2);
    float betaInCut = fasin(fmin_((-rt_InSeg * corrF + drt_tl_axis) * k2Rinv1GeVf / m.ptCut, kSinAlphaMax)) +
                      (0.02f / drt_InSeg);
    if (!(fabs_(betaInRHmin) < betaInCut))
      return false;

    float betaAv = 0.5f * (betaIn + betaOut);
    float pt_beta = drt_tl_axis * k2Rinv1GeVf / fsin(betaAv);
    int lIn = 5;
    int lOut = isEC_lastLayer ? 11 : 5;
    float sdOut_dr = segmentDr(md, q.md3, q.md4);
    float sdOut_d = md.anchorPos[q.md4].rt - md.anchorPos[q.md3].rt;
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
    const float alphaInAbsReg = fmax_(fabs_(alpha_InLo), md.slope3[q.md1]);
    const float alphaOutAbsReg = fmax_(fabs_(alpha_OutLo), md.slope3[q.md3]);
    const float dBetaInLum = lIn < 11 ? 0.0f : fabs_(alphaInAbsReg * kDeltaZLum / z_InLo);
    const float dBetaOutLum = lOut < 11 ? 0.0f : fabs_(alphaOutAbsReg * kDeltaZLum / z_OutLo);
    const float dBetaLum2 = (dBetaInLum + dBetaOutLum) * (dBetaInLum + dBetaOutLum);
    const float sinDPhi = fsin(dPhi);
    const float dBetaRIn2 = 0;
    float dBetaROut = 0;
    if (isEC_lastLayer) {
      dBetaROut = (fsqrt(md.anchorHighEdgeX[q.md4] * md.anchorHighEdgeX[q.md4] +
                         md.anchorHighEdgeY[q.md4] * md.anchorHighEdgeY[q.md4]) -
                   fsqrt(md.anchorLowEdgeX[q.md4] * md.anchorLowEdgeX[q.md4] +
                         md.anchorLowEdgeY[q.md4] * md.anchorLowEdgeY[q.md4])) *
                  sinDPhi / drt_tl_axis;
    }
    const float dBetaROut2 = dBetaROut * dBetaROut;
    float betaOutCut = fasin(fmin_(drt_tl_axis * k2Rinv1GeVf / m.ptCut, kSinAlphaMax)) + (0.02f / sdOut_d) +
                       fsqrt(dBetaLum2 + dBetaMuls * dBetaMuls);
    if (!(fabs_(betaOut) < betaOutCut))
      return false;
    float dBetaRes = 0.02f / fmin_(sdOut_d, drt_InSeg);
    return betaDifferenceCut(betaIn, betaOut, betaInRHmin, betaInRHmax, betaOutRHmin, betaOutRHmax, dBetaRes, dBetaMuls,
                             dBetaLum2, dBetaRIn2, dBetaROut2);
  }

  // Barrel-barrel-endcap-endcap and barrel-endcap-endcap-endcap
  // (SDL/Quintuplet.h:1748-2029).
  LST_HD_BIG bool t4BBEE(const Modules& m, const MiniDoublets& md, const Segments& s, const T4Input& q) {
    bool isPS_InLo = (m.moduleType[q.lmII] == PS);
    bool isPS_OutLo = (m.moduleType[q.lmOI] == PS);
    float rt_InLo = md.anchorPos[q.md1].rt, rt_InOut = md.anchorPos[q.md2].rt, rt_OutLo = md.anchorPos[q.md3].rt;
    float z_InLo = md.anchorPos[q.md1].z, z_InOut = md.anchorPos[q.md2].z, z_OutLo = md.anchorPos[q.md3].z;
    float alpha1GeV_OutLo = md.slope[q.md3];
    float dzDrtScale = md.tanSlope[q.md3] / alpha1GeV_OutLo;
    float zpitch_InLo = (isPS_InLo ? kPixelPSZpitch : kStrip2SZpitch);
    float zpitch_OutLo = (isPS_OutLo ? kPixelPSZpitch : kStrip2SZpitch);
    float zGeom = zpitch_InLo + zpitch_OutLo;
    if (!(z_InLo * z_OutLo > 0))
      return false;
    float dLum = signTransfer(kDeltaZLum, z_InLo);
    bool isOutSgInnerMDPS = m.moduleType[q.lmOI] == PS;
    float rtGeom1 = isOutSgInnerMDPS ? kPixelPSZpitch : kStrip2SZpitch;
    float zGeom1 = signTransfer(zGeom, z_InLo);
    float rtLo = rt_InLo * (1.f + (z_OutLo - z_InLo - zGeom1) / (z_InLo + zGeom1 + dLum) / dzDrtScale) - rtGeom1;
    float rtOut = rt_OutLo;
    if (!(rtOut >= rtLo))
      return false;
    float zInForHi = z_InLo - zGeom1 - dLum;
    if (zInForHi * z_InLo < 0) {
      zInForHi = signTransfer(0.1f, z_InLo);
    }
    float rtHi = rt_InLo * (1.f + (z_OutLo - z_InLo + zGeom1) / zInForHi) + rtGeom1;
    if (!((rt_OutLo >= rtLo) && (rt_OutLo <= rtHi)))
      return false;

    float rIn = fsqrt(z_InLo * z_InLo + rt_InLo * rt_InLo);
    const float drtSDIn = rt_InOut - rt_InLo;
    const float dzSDIn = z_InOut - z_InLo;
    const float dr3SDIn = fsqrt(rt_InOut * rt_InOut + z_InOut * z_InOut) - fsqrt(rt_InLo * rt_InLo + z_InLo * z_InLo);
    const float coshEta = dr3SDIn / drtSDIn;
    const float dzOutInAbs = fabs_(z_OutLo - z_InLo);
    const float multDzDr = dzOutInAbs * coshEta / (coshEta * coshEta - 1.f);
    const float zGeom1_another = kPixelPSZpitch;
    float kZ = (z_OutLo - z_InLo) / dzSDIn;
    float drtErr =
        zGeom1_another * zGeom1_another * drtSDIn * drtSDIn / dzSDIn / dzSDIn * (1.f - 2.f * kZ + 2.f * kZ * kZ);
    const float sdlThetaMulsF = 0.015f * fsqrt(0.1f + 0.2f * (rt_OutLo - rt_InLo) / 50.f) * fsqrt(rIn / rt_InLo);
    const float sdlMuls = sdlThetaMulsF * 3.f / m.ptCut * 4.f;
    drtErr += sdlMuls * sdlMuls * multDzDr * multDzDr / 3.f * coshEta * coshEta;
    drtErr = fsqrt(drtErr);
    if (!((kZ >= 0) && (rtOut >= rtLo) && (rtOut <= rtHi)))
      return false;

    const float sdlPVoff = 0.1f / rt_OutLo;
    float sdlCut = alpha1GeV_OutLo + fsqrt(sdlMuls * sdlMuls + sdlPVoff * sdlPVoff);
    float deltaPhiPos = phiMpiPi(md.anchorPhi[q.md4] - md.anchorPhi[q.md2]);
    if (!(fabs_(deltaPhiPos) <= sdlCut))
      return false;
    float midPointX = 0.5f * (md.anchorPos[q.md1].x + md.anchorPos[q.md3].x);
    float midPointY = 0.5f * (md.anchorPos[q.md1].y + md.anchorPos[q.md3].y);
    float diffX = md.anchorPos[q.md3].x - md.anchorPos[q.md1].x;
    float diffY = md.anchorPos[q.md3].y - md.anchorPos[q.md1].y;
    float dPhi = deltaPhi(midPointX, midPointY, diffX, diffY);
    if (!(fabs_(dPhi) <= sdlCut))
      return false;

    float sdIn_alpha = s.dPhiChanges[q.innerSeg];
    float sdIn_alpha_min = s.dPhiChangeMins[q.innerSeg];
    float sdIn_alpha_max = s.dPhiChangeMaxs[q.innerSeg];
    float sdOut_alpha = sdIn_alpha;
    float sdOut_alphaOut = phiMpiPi(phiOf(md.anchorPos[q.md4].x - md.anchorPos[q.md3].x, md.anchorPos[q.md4].y - md.anchorPos[q.md3].y) -
                                    md.anchorPhi[q.md4]);
    float sdOut_alphaOut_min = phiMpiPi(s.dPhiChangeMins[q.outerSeg] - s.dPhiMins[q.outerSeg]);
    float sdOut_alphaOut_max = phiMpiPi(s.dPhiChangeMaxs[q.outerSeg] - s.dPhiMaxs[q.outerSeg]);
    float tl_axis_x = md.anchorPos[q.md4].x - md.anchorPos[q.md1].x;
    float tl_axis_y = md.anchorPos[q.md4].y - md.anchorPos[q.md1].y;
    float betaIn = sdIn_alpha - phiMpiPi(phiOf(tl_axis_x, tl_axis_y) - md.anchorPhi[q.md1]);
    float betaInRHmin = betaIn;
    float betaInRHmax = betaIn;
    float betaOut = -sdOut_alphaOut + phiMpiPi(phiOf(tl_axis_x, tl_axis_y) - md.anchorPhi[q.md4]);
    float betaOutRHmin = betaOut;
    float betaOutRHmax = betaOut;
    bool isEC_secondLayer = (m.subdets[q.lmIO] == Endcap) and (m.moduleType[q.lmIO] == TwoS);
    if (isEC_secondLayer) {
      betaInRHmin = betaIn - sdIn_alpha_min + sdIn_alpha;
      betaInRHmax = betaIn - sdIn_alpha_max + sdIn_alpha;
    }
    betaOutRHmin = betaOut - sdOut_alphaOut_min + sdOut_alphaOut;
    betaOutRHmax = betaOut - sdOut_alphaOut_max + sdOut_alphaOut;
    float swapTemp;
    if (fabs_(betaOutRHmin) > fabs_(betaOutRHmax)) {
      swapTemp = betaOutRHmin;
      betaOutRHmin = betaOutRHmax;
      betaOutRHmax = swapTemp;
    }
    if (fabs_(betaInRHmin) > fabs_(betaInRHmax)) {
      swapTemp = betaInRHmin;
      betaInRHmin = betaInRHmax;
      betaInRHmax = swapTemp;
    }
    float sdIn_dr = segmentDr(md, q.md1, q.md2);
    float sdIn_d = rt_InOut - rt_InLo;
    float dr = fsqrt(tl_axis_x * tl_axis_x + tl_axis_y * tl_axis_y);
    const float corrF = 1.f;
    float betaInCut =
        fasin(fmin_((-sdIn_dr * corrF + dr) * k2Rinv1GeVf / m.ptCut, kSinAlphaMax)) + (0.02f / sdIn_d);
    if (!(fabs_(betaInRHmin) < betaInCut))
      return false;

    float betaAv = 0.5f * (betaIn + betaOut);
    float pt_beta = dr * k2Rinv1GeVf / fsin(betaAv);
    float lIn = 5;
    float lOut = 11;
    float sdOut_dr = segmentDr(md, q.md3, q.md4);
    float sdOut_d = md.anchorPos[q.md4].rt - md.anchorPos[q.md3].rt;
    deltaBetaIterations(betaIn, betaOut, betaAv, pt_beta, sdIn_dr, sdOut_dr, dr, lIn);

    const float betaInMMSF =
        (fabs_(betaInRHmin + betaInRHmax) > 0) ? (2.f * betaIn / fabs_(betaInRHmin + betaInRHmax)) : 0.f;
    const float betaOutMMSF =
        (fabs_(betaOutRHmin + betaOutRHmax) > 0) ? (2.f * betaOut / fabs_(betaOutRHmin + betaOutRHmax)) : 0.f;
    betaInRHmin *= betaInMMSF;
    betaInRHmax *= betaInMMSF;
    betaOutRHmin *= betaOutMMSF;
    betaOutRHmax *= betaOutMMSF;

    const float dBetaMuls = sdlThetaMulsF * 4.f / fmin_(fabs_(pt_beta), kPtBetaMax);
    const float alphaInAbsReg = fmax_(fabs_(sdIn_alpha), md.slope3[q.md1]);
    const float alphaOutAbsReg = fmax_(fabs_(sdOut_alpha), md.slope3[q.md3]);
    const float dBetaInLum = lIn < 11 ? 0.0f : fabs_(alphaInAbsReg * kDeltaZLum / z_InLo);
    const float dBetaOutLum = lOut < 11 ? 0.0f : fabs_(alphaOutAbsReg * kDeltaZLum / z_OutLo);
    const float dBetaLum2 = (dBetaInLum + dBetaOutLum) * (dBetaInLum + dBetaOutLum);
    const float sinDPhi = fsin(dPhi);
    const float dBetaRIn2 = 0;
    float dBetaROut = 0;
    if (m.moduleType[q.lmOO] == TwoS) {
      dBetaROut = (fsqrt(md.anchorHighEdgeX[q.md4] * md.anchorHighEdgeX[q.md4] +
                         md.anchorHighEdgeY[q.md4] * md.anchorHighEdgeY[q.md4]) -
                   fsqrt(md.anchorLowEdgeX[q.md4] * md.anchorLowEdgeX[q.md4] +
                         md.anchorLowEdgeY[q.md4] * md.anchorLowEdgeY[q.md4])) *
                  sinDPhi / dr;
    }
    const float dBetaROut2 = dBetaROut * dBetaROut;
    float betaOutCut = fasin(fmin_(dr * k2Rinv1GeVf / m.ptCut, kSinAlphaMax)) + (0.02f / sdOut_d) +
                       fsqrt(dBetaLum2 + dBetaMuls * dBetaMuls);
    if (!(fabs_(betaOut) < betaOutCut))
      return false;
    float dBetaRes = 0.02f / fmin_(sdOut_d, sdIn_d);
    return betaDifferenceCut(betaIn, betaOut, betaInRHmin, betaInRHmax, betaOutRHmin, betaOutRHmax, dBetaRes, dBetaMuls,
                             dBetaLum2, dBetaRIn2, dBetaROut2);
  }

  // Endcap-endcap-endcap-endcap (SDL/Quintuplet.h:2031-2297).
  LST_HD_BIG bool t4EEEE(const Modules& m, const MiniDoublets& md, const Segments& s, const T4Input& q) {
    float rt_InLo = md.anchorPos[q.md1].rt, rt_InOut = md.anchorPos[q.md2].rt, rt_OutLo = md.anchorPos[q.md3].rt;
    float z_InLo = md.anchorPos[q.md1].z, z_InOut = md.anchorPos[q.md2].z, z_OutLo = md.anchorPos[q.md3].z;
    float alpha1GeV_OutLo = md.slope[q.md3];
    float dzDrtScale = md.tanSlope[q.md3] / alpha1GeV_OutLo;
    if (!((z_InLo * z_OutLo) > 0))
      return false;
    float dLum = signTransfer(kDeltaZLum, z_InLo);
    bool isOutSgInnerMDPS = m.moduleType[q.lmOI] == PS;
    bool isInSgInnerMDPS = m.moduleType[q.lmII] == PS;
    float rtGeom = (isInSgInnerMDPS and isOutSgInnerMDPS)  ? 2.f * kPixelPSZpitch
                   : (isInSgInnerMDPS or isOutSgInnerMDPS) ? kPixelPSZpitch + kStrip2SZpitch
                                                           : 2.f * kStrip2SZpitch;
    float dz = z_OutLo - z_InLo;
    float rtLo = rt_InLo * (1.f + dz / (z_InLo + dLum) / dzDrtScale) - rtGeom;
    float rtOut = rt_OutLo;
    float rtHi = rt_InLo * (1.f + dz / (z_InLo - dLum)) + rtGeom;
    if (!((rtOut >= rtLo) && (rtOut <= rtHi)))
      return false;

    bool isInSgOuterMDPS = m.moduleType[q.lmIO] == PS;
    const float drtSDIn = rt_InOut - rt_InLo;
    const float dzSDIn = z_InOut - z_InLo;
    const float dr3SDIn = fsqrt(rt_InOut * rt_InOut + z_InOut * z_InOut) - fsqrt(rt_InLo * rt_InLo + z_InLo * z_InLo);
    float coshEta = dr3SDIn / drtSDIn;
    float dzOutInAbs = fabs_(z_OutLo - z_InLo);
    float multDzDr = dzOutInAbs * coshEta / (coshEta * coshEta - 1.f);
    float kZ = (z_OutLo - z_InLo) / dzSDIn;
    float sdlThetaMulsF = 0.015f * fsqrt(0.1f + 0.2f * (rt_OutLo - rt_InLo) / 50.f);
    float sdlMuls = sdlThetaMulsF * 3.f / m.ptCut * 4.f;
    float drtErr = fsqrt(kPixelPSZpitch * kPixelPSZpitch * 2.f / (dzSDIn * dzSDIn) * (dzOutInAbs * dzOutInAbs) +
                         sdlMuls * sdlMuls * multDzDr * multDzDr / 3.f * coshEta * coshEta);
    float drtMean = drtSDIn * dzOutInAbs / fabs_(dzSDIn);
    float rtWindow = drtErr + rtGeom;
    float rtLo_point = rt_InLo + drtMean / dzDrtScale - rtWindow;
    float rtHi_point = rt_InLo + drtMean + rtWindow;
    if (isInSgInnerMDPS and isInSgOuterMDPS) {
      if (!(kZ >= 0 and rtOut >= rtLo_point and rtOut <= rtHi_point))
        return false;
    }

    float sdlPVoff = 0.1f / rtOut;
    float sdlCut = alpha1GeV_OutLo + fsqrt(sdlMuls * sdlMuls + sdlPVoff * sdlPVoff);
    float deltaPhiPos = phiMpiPi(md.anchorPhi[q.md4] - md.anchorPhi[q.md2]);
    if (!(fabs_(deltaPhiPos) <= sdlCut))
      return false;
    float midPointX = 0.5f * (md.anchorPos[q.md1].x + md.anchorPos[q.md3].x);
    float midPointY = 0.5f * (md.anchorPos[q.md1].y + md.anchorPos[q.md3].y);
    float diffX = md.anchorPos[q.md3].x - md.anchorPos[q.md1].x;
    float diffY = md.anchorPos[q.md3].y - md.anchorPos[q.md1].y;
    float dPhi = deltaPhi(midPointX, midPointY, diffX, diffY);
    if (!((fabs_(dPhi) <= sdlCut)))
      return false;

    float sdIn_alpha = s.dPhiChanges[q.innerSeg];
    float sdOut_alpha = sdIn_alpha;
    float sdOut_dPhiPos = phiMpiPi(md.anchorPhi[q.md4] - md.anchorPhi[q.md3]);
    float sdOut_dPhiChange = s.dPhiChanges[q.outerSeg];
    float sdOut_dPhiChange_min = s.dPhiChangeMins[q.outerSeg];
    float sdOut_dPhiChange_max = s.dPhiChangeMaxs[q.outerSeg];
    float sdOut_alphaOutRHmin = phiMpiPi(sdOut_dPhiChange_min - sdOut_dPhiPos);
    float sdOut_alphaOutRHmax = phiMpiPi(sdOut_dPhiChange_max - sdOut_dPhiPos);
    float sdOut_alphaOut = phiMpiPi(sdOut_dPhiChange - sdOut_dPhiPos);
    float tl_axis_x = md.anchorPos[q.md4].x - md.anchorPos[q.md1].x;
    float tl_axis_y = md.anchorPos[q.md4].y - md.anchorPos[q.md1].y;
    float betaIn = sdIn_alpha - phiMpiPi(phiOf(tl_axis_x, tl_axis_y) - md.anchorPhi[q.md1]);
    float sdIn_alphaRHmin = s.dPhiChangeMins[q.innerSeg];
    float sdIn_alphaRHmax = s.dPhiChangeMaxs[q.innerSeg];
    float betaInRHmin = betaIn + sdIn_alphaRHmin - sdIn_alpha;
    float betaInRHmax = betaIn + sdIn_alphaRHmax - sdIn_alpha;
    float betaOut = -sdOut_alphaOut + phiMpiPi(phiOf(tl_axis_x, tl_axis_y) - md.anchorPhi[q.md4]);
    float betaOutRHmin = betaOut - sdOut_alphaOutRHmin + sdOut_alphaOut;
    float betaOutRHmax = betaOut - sdOut_alphaOutRHmax + sdOut_alphaOut;
    float swapTemp;
    if (fabs_(betaOutRHmin) > fabs_(betaOutRHmax)) {
      swapTemp = betaOutRHmin;
      betaOutRHmin = betaOutRHmax;
      betaOutRHmax = swapTemp;
    }
    if (fabs_(betaInRHmin) > fabs_(betaInRHmax)) {
      swapTemp = betaInRHmin;
      betaInRHmin = betaInRHmax;
      betaInRHmax = swapTemp;
    }
    float sdIn_dr = segmentDr(md, q.md1, q.md2);
    float sdIn_d = rt_InOut - rt_InLo;
    float dr = fsqrt(tl_axis_x * tl_axis_x + tl_axis_y * tl_axis_y);
    const float corrF = 1.f;
    float betaInCut =
        fasin(fmin_((-sdIn_dr * corrF + dr) * k2Rinv1GeVf / m.ptCut, kSinAlphaMax)) + (0.02f / sdIn_d);
    if (!(fabs_(betaInRHmin) < betaInCut))
      return false;

    float betaAv = 0.5f * (betaIn + betaOut);
    float pt_beta = dr * k2Rinv1GeVf / fsin(betaAv);
    int lIn = 11;
    int lOut = 13;
    float sdOut_dr = segmentDr(md, q.md3, q.md4);
    float sdOut_d = md.anchorPos[q.md4].rt - md.anchorPos[q.md3].rt;
    deltaBetaIterations(betaIn, betaOut, betaAv, pt_beta, sdIn_dr, sdOut_dr, dr, lIn);

    const float betaInMMSF =
        (fabs_(betaInRHmin + betaInRHmax) > 0) ? (2.f * betaIn / fabs_(betaInRHmin + betaInRHmax)) : 0.f;
    const float betaOutMMSF =
        (fabs_(betaOutRHmin + betaOutRHmax) > 0) ? (2.f * betaOut / fabs_(betaOutRHmin + betaOutRHmax)) : 0.f;
    betaInRHmin *= betaInMMSF;
    betaInRHmax *= betaInMMSF;
    betaOutRHmin *= betaOutMMSF;
    betaOutRHmax *= betaOutMMSF;

    const float dBetaMuls = sdlThetaMulsF * 4.f / fmin_(fabs_(pt_beta), kPtBetaMax);
    const float alphaInAbsReg = fmax_(fabs_(sdIn_alpha), md.slope3[q.md1]);
    const float alphaOutAbsReg = fmax_(fabs_(sdOut_alpha), md.slope3[q.md3]);
    const float dBetaInLum = lIn < 11 ? 0.0f : fabs_(alphaInAbsReg * kDeltaZLum / z_InLo);
    const float dBetaOutLum = lOut < 11 ? 0.0f : fabs_(alphaOutAbsReg * kDeltaZLum / z_OutLo);
    const float dBetaLum2 = (dBetaInLum + dBetaOutLum) * (dBetaInLum + dBetaOutLum);
    const float dBetaRIn2 = 0;
    float dBetaROut2 = 0;
    float betaOutCut = fasin(fmin_(dr * k2Rinv1GeVf / m.ptCut, kSinAlphaMax)) + (0.02f / sdOut_d) +
                       fsqrt(dBetaLum2 + dBetaMuls * dBetaMuls);
    if (!(fabs_(betaOut) < betaOutCut))
      return false;
    float dBetaRes = 0.02f / fmin_(sdOut_d, sdIn_d);
    return betaDifferenceCut(betaIn, betaOut, betaInRHmin, betaInRHmax, betaOutRHmin, betaOutRHmax, dBetaRes, dBetaMuls,
                             dBetaLum2, dBetaRIn2, dBetaROut2);
  }

  // Dispatch on the subdetectors of the four modules (SDL/Quintuplet.h:2299-2506).
  LST_HD bool t4Select(const Modules& m, const MiniDoublets& md, const Segments& s, const T4Input& q) {
    short a = m.subdets[q.lmII], b = m.subdets[q.lmIO], c = m.subdets[q.lmOI], d = m.subdets[q.lmOO];
    if (a == Barrel and b == Barrel and c == Barrel and d == Barrel)
      return t4BBBB(m, md, s, q);
    if (a == Barrel and b == Barrel and c == Endcap and d == Endcap)
      return t4BBEE(m, md, s, q);
    if (a == Barrel and b == Barrel and c == Barrel and d == Endcap)
      return t4BBBB(m, md, s, q);
    if (a == Barrel and b == Endcap and c == Endcap and d == Endcap)
      return t4BBEE(m, md, s, q);
    if (a == Endcap and b == Endcap and c == Endcap and d == Endcap)
      return t4EEEE(m, md, s, q);
    return false;
  }

  // ------------------------------------------------------- radius checks
  // Spread of the circle radius when 2S endcap hits move along their strips
  // (SDL/Quintuplet.h:753-783).
  // Min and max circle radius over the 3 x 3 x 3 choices of the three points'
  // positions (SDL/Quintuplet.h:753-783).  n1..n3 = 1 for a point whose three
  // candidate positions coincide: repeated candidates leave fmin / fmax
  // unchanged, so the result equals the full 27-fit loop.
  LST_HD void radiusSpread(const float* x1, const float* y1, int n1, const float* x2, const float* y2, int n2,
                           const float* x3, const float* y3, int n3, float& minimumRadius, float& maximumRadius) {
    float g, f;
    minimumRadius = kInf;
    maximumRadius = 0.f;
    for (int i = 0; i < n1; i++)
      for (int j = 0; j < n2; j++)
        for (int k = 0; k < n3; k++) {
          float candidateRadius = circleFrom3(x1[i], y1[i], x2[j], y2[j], x3[k], y3[k], g, f);
          maximumRadius = fmax_(candidateRadius, maximumRadius);
          minimumRadius = fmin_(candidateRadius, minimumRadius);
        }
  }

  // Inverse-radius compatibility of the inner and bridge circles
  // (SDL/Quintuplet.h:785-1133).  kind: 0 BBBBB, 1 BBBBE, 2 BBBEE(layer 1),
  // 3 BBBEE(layer 2), 4 BBBEE(other), 5 BBEEE, 6 BEEEE, 7 EEEEE.
  LST_HD bool matchRadii(int kind,
                         float innerRadius,
                         float bridgeRadius,
                         float innerRadiusMin2S,
                         float innerRadiusMax2S,
                         float bridgeRadiusMin2S,
                         float bridgeRadiusMax2S) {
    float eIn, eBr;
    const bool highPt = innerRadius > 2.0f / (2.f * k2Rinv1GeVf);
    switch (kind) {
      case 0:
        eIn = highPt ? 0.4449f : 0.1512f;
        eBr = highPt ? 0.4033f : 0.1781f;
        break;
      case 1:
        eIn = highPt ? 0.4750f : 0.1781f;
        eBr = highPt ? 0.3903f : 0.2167f;
        break;
      case 2:
        eIn = 0.178f;
        eBr = 0.507f;
        break;
      case 3:
        eIn = 0.2097f;
        eBr = 0.8557f;
        break;
      case 4:
        eIn = 0.066f;
        eBr = 0.617f;
        break;
      case 5:
        eIn = highPt ? 12.9173f : 0.6376f;
        eBr = highPt ? 5.1700f : 2.1381f;
        break;
      case 6:
        eIn = highPt ? 23.2713f : 1.9382f;
        eBr = highPt ? 21.7980f : 3.7280f;
        break;
      default:
        eIn = highPt ? 22.5226f : 1.9382f;
        eBr = highPt ? 21.0966f : 2.2091f;
        break;
    }
    float innerInvRadiusMax = (1.f + eIn) / innerRadius;
    float innerInvRadiusMin = fmax_(0.f, (1.f - eIn) / innerRadius);
    float bridgeInvRadiusMax = (1.f + eBr) / bridgeRadius;
    float bridgeInvRadiusMin = fmax_(0.f, (1.f - eBr) / bridgeRadius);
    if (kind <= 1)
      return intervalsOverlap(innerInvRadiusMin, innerInvRadiusMax, bridgeInvRadiusMin, bridgeInvRadiusMax);
    if (kind <= 5)
      return intervalsOverlap(innerInvRadiusMin,
                              innerInvRadiusMax,
                              fmin_(bridgeInvRadiusMin, 1.0f / bridgeRadiusMax2S),
                              fmax_(bridgeInvRadiusMax, 1.0f / bridgeRadiusMin2S));
    // The reference forms these four bounds in double precision.
    return intervalsOverlap(static_cast<float>(fmin_(innerInvRadiusMin, 1.0 / innerRadiusMax2S)),
                            static_cast<float>(fmax_(innerInvRadiusMax, 1.0 / innerRadiusMin2S)),
                            static_cast<float>(fmin_(bridgeInvRadiusMin, 1.0 / bridgeRadiusMax2S)),
                            static_cast<float>(fmax_(bridgeInvRadiusMax, 1.0 / bridgeRadiusMin2S)));
  }

  // --------------------------------------------------------- r-z chi-square
  // Helix r-z residuals of the outer hits (SDL/Quintuplet.h:302-736); sets
  // tightCutFlag for the T5-in-TC selection.
  LST_HD_BIG bool t5PassRZ(const Modules& m,
                       const MiniDoublets& md,
                       const unsigned int* mdIdx,
                       const uint16_t* lm,
                       float& rzChiSquared,
                       float inner_pt,
                       float innerRadius,
                       float g,
                       float f,
                       bool& tightCutFlag) {
    const float rt1 = md.anchorPos[mdIdx[0]].rt / 100, rt2 = md.anchorPos[mdIdx[1]].rt / 100, rt3 = md.anchorPos[mdIdx[2]].rt / 100,
                rt4 = md.anchorPos[mdIdx[3]].rt / 100, rt5 = md.anchorPos[mdIdx[4]].rt / 100;
    const float z1 = md.anchorPos[mdIdx[0]].z / 100, z2 = md.anchorPos[mdIdx[1]].z / 100, z3 = md.anchorPos[mdIdx[2]].z / 100,
                z4 = md.anchorPos[mdIdx[3]].z / 100, z5 = md.anchorPos[mdIdx[4]].z / 100;
    const int layer1 = m.sdlLayers[lm[0]], layer2 = m.sdlLayers[lm[1]], layer3 = m.sdlLayers[lm[2]],
              layer4 = m.sdlLayers[lm[3]], layer5 = m.sdlLayers[lm[4]];
    const int moduleType1 = m.moduleType[lm[0]], moduleType2 = m.moduleType[lm[1]], moduleType3 = m.moduleType[lm[2]],
              moduleType4 = m.moduleType[lm[3]], moduleType5 = m.moduleType[lm[4]];
    const float x1 = md.anchorPos[mdIdx[0]].x / 100, x2 = md.anchorPos[mdIdx[1]].x / 100, x3 = md.anchorPos[mdIdx[2]].x / 100,
                x4 = md.anchorPos[mdIdx[3]].x / 100;
    const float y1 = md.anchorPos[mdIdx[0]].y / 100, y2 = md.anchorPos[mdIdx[1]].y / 100, y3 = md.anchorPos[mdIdx[2]].y / 100,
                y4 = md.anchorPos[mdIdx[3]].y / 100;

    float residual = 0;
    float error = 0;
    float x_center = g / 100, y_center = f / 100;
    float x_init = md.anchorPos[mdIdx[2]].x / 100;
    float y_init = md.anchorPos[mdIdx[2]].y / 100;
    float z_init = md.anchorPos[mdIdx[2]].z / 100;
    float rt_init = md.anchorPos[mdIdx[2]].rt / 100;
    if (moduleType3 == 1) {
      x_init = md.anchorPos[mdIdx[1]].x / 100;
      y_init = md.anchorPos[mdIdx[1]].y / 100;
      z_init = md.anchorPos[mdIdx[1]].z / 100;
      rt_init = md.anchorPos[mdIdx[1]].rt / 100;
    }

    int charge = 0;
    float slope3c = (y3 - y_center) / (x3 - x_center);
    float slope1c = (y1 - y_center) / (x1 - x_center);
    if ((y3 - y_center) > 0 && (y1 - y_center) > 0) {
      if (slope1c > 0 && slope3c < 0)
        charge = -1;
      else if (slope1c < 0 && slope3c > 0)
        charge = 1;
      else if (slope3c > slope1c)
        charge = -1;
      else if (slope3c < slope1c)
        charge = 1;
    } else if ((y3 - y_center) < 0 && (y1 - y_center) < 0) {
      if (slope1c < 0 && slope3c > 0)
        charge = 1;
      else if (slope1c > 0 && slope3c < 0)
        charge = -1;
      else if (slope3c > slope1c)
        charge = -1;
      else if (slope3c < slope1c)
        charge = 1;
    } else if ((y3 - y_center) < 0 && (y1 - y_center) > 0) {
      if ((x3 - x_center) > 0 && (x1 - x_center) > 0)
        charge = 1;
      else if ((x3 - x_center) < 0 && (x1 - x_center) < 0)
        charge = -1;
    } else if ((y3 - y_center) > 0 && (y1 - y_center) < 0) {
      if ((x3 - x_center) > 0 && (x1 - x_center) > 0)
        charge = -1;
      else if ((x3 - x_center) < 0 && (x1 - x_center) < 0)
        charge = 1;
    }

    float pseudo_phi = fatan((y_init - y_center) / (x_init - x_center));
    float Pt = inner_pt;
    float Px = Pt * fabs_(fsin(pseudo_phi));
    // The reference writes an unqualified cos() here, which resolves to the
    // double-precision C function: Py is formed in double and rounded once.
    float Py = static_cast<float>(Pt * fabs_(::cos(static_cast<double>(pseudo_phi))));

    if (x_init > x_center && y_init > y_center) {
      if (charge == 1)
        Py = -Py;
      if (charge == -1)
        Px = -Px;
    }
    if (x_init < x_center && y_init > y_center) {
      if (charge == -1) {
        Px = -Px;
        Py = -Py;
      }
    }
    if (x_init < x_center && y_init < y_center) {
      if (charge == 1)
        Px = -Px;
      if (charge == -1)
        Py = -Py;
    }
    if (x_init > x_center && y_init < y_center) {
      if (charge == 1) {
        Px = -Px;
        Py = -Py;
      }
    }
    if (moduleType3 == 0) {
      if (x4 < x3 && x3 < x2)
        Px = -fabs_(Px);
      if (x4 > x3 && x3 > x2)
        Px = fabs_(Px);
      if (y4 < y3 && y3 < y2)
        Py = -fabs_(Py);
      if (y4 > y3 && y3 > y2)
        Py = fabs_(Py);
    } else if (moduleType3 == 1) {
      if (x3 < x2 && x2 < x1)
        Px = -fabs_(Px);
      if (x3 > x2 && x2 > x1)
        Px = fabs_(Px);
      if (y3 < y2 && y2 < y1)
        Py = -fabs_(Py);
      if (y3 > y2 && y2 > y1)
        Py = fabs_(Py);
    }

    float AO = fsqrt((x1 - x_center) * (x1 - x_center) + (y1 - y_center) * (y1 - y_center));
    float BO = fsqrt((x_init - x_center) * (x_init - x_center) + (y_init - y_center) * (y_init - y_center));
    float AB = fsqrt((x1 - x_init) * (x1 - x_init) + (y1 - y_init) * (y1 - y_init));
    float dPhi = facos((AO * AO + BO * BO - AB * AB) / (2 * AO * BO));
    float ds = innerRadius / 100 * dPhi;
    float Pz = (z_init - z1) / ds * Pt;
    float p = fsqrt(Px * Px + Py * Py + Pz * Pz);
    float Bz = kMagneticField;
    float a = -0.299792 * Bz * charge;

    float zsi = 0, rtsi = 0;
    int layeri = 0, moduleTypei = 0;
    rzChiSquared = 0;
    for (int i = 2; i < 6; i++) {
      if (i == 2) {
        zsi = z2;
        rtsi = rt2;
        layeri = layer2;
        moduleTypei = moduleType2;
      } else if (i == 3) {
        zsi = z3;
        rtsi = rt3;
        layeri = layer3;
        moduleTypei = moduleType3;
      } else if (i == 4) {
        zsi = z4;
        rtsi = rt4;
        layeri = layer4;
        moduleTypei = moduleType4;
      } else {
        zsi = z5;
        rtsi = rt5;
        layeri = layer5;
        moduleTypei = moduleType5;
      }
      if (moduleType3 == 0) {
        if (i == 3)
          continue;
      } else {
        if (i == 2)
          continue;
      }
      float diffr = 0, diffz = 0;
      float rou = a / p;
      float s = (zsi - z_init) * p / Pz;
      float x = x_init + Px / a * fsin(rou * s) - Py / a * (1 - fcos(rou * s));
      float y = y_init + Py / a * fsin(rou * s) + Px / a * (1 - fcos(rou * s));
      diffr = (rtsi - fsqrt(x * x + y * y)) * 100;
      if (layeri <= 6) {
        float paraA = rt_init * rt_init + 2 * (Px * Px + Py * Py) / (a * a) + 2 * (y_init * Px - x_init * Py) / a -
                      rtsi * rtsi;
        float paraB = 2 * (x_init * Px + y_init * Py) / a;
        float paraC = 2 * (y_init * Px - x_init * Py) / a + 2 * (Px * Px + Py * Py) / (a * a);
        float A = paraB * paraB + paraC * paraC;
        float B = 2 * paraA * paraB;
        float C = paraA * paraA - paraC * paraC;
        float sol1 = (-B + fsqrt(B * B - 4 * A * C)) / (2 * A);
        float sol2 = (-B - fsqrt(B * B - 4 * A * C)) / (2 * A);
        float solz1 = fasin(sol1) / rou * Pz / p + z_init;
        float solz2 = fasin(sol2) / rou * Pz / p + z_init;
        float diffz1 = (solz1 - zsi) * 100;
        float diffz2 = (solz2 - zsi) * 100;
        if (fisnan(diffz1))
          diffz = diffz2;
        else if (fisnan(diffz2))
          diffz = diffz1;
        else
          diffz = (fabs_(diffz1) < fabs_(diffz2)) ? diffz1 : diffz2;
      }
      residual = (layeri > 6) ? diffr : diffz;
      if (moduleTypei == 0)
        error = 0.15f;
      else
        error = 5.0f;
      if (i == 2 || i == 3) {
        uint16_t lmi = (i == 2) ? lm[1] : lm[2];
        float drdz = fabs_(m.drdzs[lmi]);
        short side = m.sides[lmi];
        short subdets = m.subdets[lmi];
        residual = (layeri <= 6 && ((side == Center) or (drdz < 1))) ? diffz : diffr;
        float projection_missing = 1;
        if (drdz < 1)
          projection_missing = ((subdets == Endcap) or (side == Center)) ? 1.f : 1 / fsqrt(1 + drdz * drdz);
        if (drdz > 1)
          projection_missing = ((subdets == Endcap) or (side == Center)) ? 1.f : drdz / fsqrt(1 + drdz * drdz);
        error = error * projection_missing;
      }
      rzChiSquared += 12 * (residual * residual) / (error * error);
    }

    if (inner_pt > 100 || fisnan(rzChiSquared)) {
      float slope;
      if (moduleType1 == 0 and moduleType2 == 0 and moduleType3 == 1)
        slope = (z2 - z1) / (rt2 - rt1);
      else
        slope = (z3 - z1) / (rt3 - rt1);
      float residual4_linear = (layer4 <= 6) ? ((z4 - z1) - slope * (rt4 - rt1)) : ((rt4 - rt1) - (z4 - z1) / slope);
      float residual5_linear = (layer4 <= 6) ? ((z5 - z1) - slope * (rt5 - rt1)) : ((rt5 - rt1) - (z5 - z1) / slope);
      residual4_linear = (moduleType4 == 0) ? residual4_linear / 0.15f : residual4_linear / 5.0f;
      residual5_linear = (moduleType5 == 0) ? residual5_linear / 0.15f : residual5_linear / 5.0f;
      residual4_linear = residual4_linear * 100;
      residual5_linear = residual5_linear * 100;
      rzChiSquared = 12 * (residual4_linear * residual4_linear + residual5_linear * residual5_linear);
      return rzChiSquared < 4.677f;
    }

    tightCutFlag = false;
    const float c = rzChiSquared;
    if (layer1 == 7 and layer2 == 8 and layer3 == 9 and layer4 == 10 and layer5 == 11) {
      if (c < 94.470f)
        tightCutFlag = true;
      return true;
    } else if (layer1 == 7 and layer2 == 8 and layer3 == 9 and layer4 == 10 and layer5 == 16) {
      if (c < 22.099f)
        tightCutFlag = true;
      return c < 37.956f;
    } else if (layer1 == 7 and layer2 == 8 and layer3 == 9 and layer4 == 15 and layer5 == 16) {
      if (c < 7.992f)
        tightCutFlag = true;
      return c < 11.622f;
    } else if (layer1 == 1 and layer2 == 7 and layer3 == 8 and layer4 == 9) {
      if (layer5 == 10) {
        if (c < 111.390f)
          tightCutFlag = true;
        return true;
      }
      if (layer5 == 15) {
        if (c < 18.351f)
          tightCutFlag = true;
        return c < 37.941f;
      }
    } else if (layer1 == 1 and layer2 == 2 and layer3 == 7) {
      if (layer4 == 8 and layer5 == 9) {
        if (c < 116.148f)
          tightCutFlag = true;
        return true;
      }
      if (layer4 == 8 and layer5 == 14) {
        if (c < 19.352f)
          tightCutFlag = true;
        return c < 52.561f;
      } else if (layer4 == 13 and layer5 == 14) {
        if (c < 10.392f)
          tightCutFlag = true;
        return c < 13.76f;
      }
    } else if (layer1 == 1 and layer2 == 2 and layer3 == 3) {
      if (layer4 == 7 and layer5 == 8) {
        if (c < 27.824f)
          tightCutFlag = true;
        return c < 44.247f;
      } else if (layer4 == 7 and layer5 == 13) {
        if (c < 18.145f)
          tightCutFlag = true;
        return c < 33.752f;
      } else if (layer4 == 12 and layer5 == 13) {
        if (c < 13.308f)
          tightCutFlag = true;
        return c < 21.213f;
      } else if (layer4 == 4 and layer5 == 5) {
        if (c < 15.627f)
          tightCutFlag = true;
        return c < 29.035f;
      } else if (layer4 == 4 and layer5 == 12) {
        if (c < 14.64f)
          tightCutFlag = true;
        return c < 23.037f;
      }
    } else if (layer1 == 2 and layer2 == 7 and layer3 == 8) {
      if (layer4 == 9 and layer5 == 15) {
        if (c < 24.662f)
          tightCutFlag = true;
        return c < 41.036f;
      } else if (layer4 == 14 and layer5 == 15) {
        if (c < 8.866f)
          tightCutFlag = true;
        return c < 14.092f;
      }
    } else if (layer1 == 2 and layer2 == 3 and layer3 == 7) {
      if (layer4 == 8 and layer5 == 14) {
        if (c < 23.730f)
          tightCutFlag = true;
        return c < 23.748f;
      }
      if (layer4 == 13 and layer5 == 14) {
        if (c < 10.772f)
          tightCutFlag = true;
        return c < 17.945f;
      }
    } else if (layer1 == 2 and layer2 == 3 and layer3 == 4) {
      if (layer4 == 5 and layer5 == 6) {
        if (c < 6.065f)
          tightCutFlag = true;
        return c < 8.803f;
      } else if (layer4 == 5 and layer5 == 12) {
        if (c < 5.693f)
          tightCutFlag = true;
        return c < 7.930f;
      } else if (layer4 == 12 and layer5 == 13) {
        if (c < 5.473f)
          tightCutFlag = true;
        return c < 7.626f;
      }
    }
    return true;
  }

  // r-phi chi-squared cut of the cut-only method (SDL/Quintuplet.h:218-300).
  LST_HD bool t5PassRPhiChi2(const Modules& m, const uint16_t* lm, float chiSquared) {
    const int layer1 = m.sdlLayers[lm[0]], layer2 = m.sdlLayers[lm[1]], layer3 = m.sdlLayers[lm[2]],
              layer4 = m.sdlLayers[lm[3]], layer5 = m.sdlLayers[lm[4]];
    if (layer1 == 7 and layer2 == 8 and layer3 == 9) {
      if (layer4 == 10 and layer5 == 11) {
        return chiSquared < 0.01788f;
      } else if (layer4 == 10 and layer5 == 16) {
        return chiSquared < 0.04725f;
      } else if (layer4 == 15 and layer5 == 16) {
        return chiSquared < 0.04725f;
      }
    } else if (layer1 == 1 and layer2 == 7 and layer3 == 8) {
      if (layer4 == 9 and layer5 == 10) {
        return chiSquared < 0.01788f;
      } else if (layer4 == 9 and layer5 == 15) {
        return chiSquared < 0.08234f;
      }
    } else if (layer1 == 1 and layer2 == 2 and layer3 == 7) {
      if (layer4 == 8 and layer5 == 9) {
        return chiSquared < 0.02360f;
      } else if (layer4 == 8 and layer5 == 14) {
        return chiSquared < 0.07167f;
      } else if (layer4 == 13 and layer5 == 14) {
        return chiSquared < 0.08234f;
      }
    } else if (layer1 == 1 and layer2 == 2 and layer3 == 3) {
      if (layer4 == 7 and layer5 == 8) {
        return chiSquared < 0.01026f;
      } else if (layer4 == 7 and layer5 == 13) {
        return chiSquared < 0.06238f;
      } else if (layer4 == 12 and layer5 == 13) {
        return chiSquared < 0.06238f;
      }
    } else if (layer1 == 1 and layer2 == 2 and layer3 == 3 and layer4 == 4) {
      if (layer5 == 5) {
        return chiSquared < 0.04725f;
      } else if (layer5 == 12) {
        return chiSquared < 0.09461f;
      }
    } else if (layer1 == 2 and layer2 == 7 and layer3 == 8) {
      if (layer4 == 9 and layer5 == 10) {
        return chiSquared < 0.00512f;
      }
      if (layer4 == 9 and layer5 == 15) {
        return chiSquared < 0.04112f;
      } else if (layer4 == 14 and layer5 == 15) {
        return chiSquared < 0.06238f;
      }
    } else if (layer1 == 2 and layer2 == 3 and layer3 == 7) {
      if (layer4 == 8 and layer5 == 14) {
        return chiSquared < 0.07167f;
      } else if (layer4 == 13 and layer5 == 14) {
        return chiSquared < 0.06238f;
      }
    } else if (layer1 == 2 and layer2 == 3 and layer3 == 4) {
      if (layer4 == 5 and layer5 == 6) {
        return chiSquared < 0.08234f;
      } else if (layer4 == 5 and layer5 == 12) {
        return chiSquared < 0.10870f;
      } else if (layer4 == 12 and layer5 == 13) {
        return chiSquared < 0.10870f;
      }
    } else if (layer1 == 3 and layer2 == 7 and layer3 == 8 and layer4 == 14 and layer5 == 15) {
      return chiSquared < 0.09461f;
    } else if (layer1 == 3 and layer2 == 4 and layer3 == 5 and layer4 == 12 and layer5 == 13) {
      return chiSquared < 0.09461f;
    }
    return true;
  }

  // --------------------------------------------------- circle regression
  // Per-hit resolution model (SDL/Quintuplet.h:1136-1221).
  LST_HD_BIG void regressionSigmas(const Modules& m,
                               const uint16_t* lm,
                               float* delta1,
                               float* delta2,
                               float* slopes,
                               bool* isFlat,
                               int nPoints,
                               bool anchorHits) {
    float inv1 = 0.01f / 0.009f;
    float inv2 = 0.15f / 0.009f;
    float inv3 = 2.4f / 0.009f;
    for (int i = 0; i < nPoints; i++) {
      uint8_t moduleType = m.moduleType[lm[i]];
      short moduleSubdet = m.subdets[lm[i]];
      short moduleSide = m.sides[lm[i]];
      const float drdz = m.drdzs[lm[i]];
      slopes[i] = m.dxdys[lm[i]];
      if (moduleSubdet == Barrel and moduleType == PS and moduleSide == Center) {
        delta1[i] = inv1;
        delta2[i] = inv1;
        slopes[i] = -999.f;
        isFlat[i] = true;
      } else if (moduleSubdet == Barrel and moduleType == TwoS) {
        delta1[i] = 1.f;
        delta2[i] = 1.f;
        slopes[i] = -999.f;
        isFlat[i] = true;
      } else if (moduleSubdet == Barrel and moduleType == PS and moduleSide != Center) {
        delta1[i] = inv1;
        isFlat[i] = false;
        if (anchorHits)
          delta2[i] = (inv2 * drdz / fsqrt(1 + drdz * drdz));
        else
          delta2[i] = (inv3 * drdz / fsqrt(1 + drdz * drdz));
      } else if (moduleSubdet == Endcap and moduleType == PS) {
        delta1[i] = inv1;
        isFlat[i] = false;
        delta2[i] = anchorHits ? inv2 : inv3;
      } else if (moduleSubdet == Endcap and moduleType == TwoS) {
        delta1[i] = 1.f;
        delta2[i] = 500.f * inv1;
        isFlat[i] = false;
      }
    }
  }

  // Rotation angle of a hit's measurement frame (shared by the fits below).
  LST_HD void measurementFrame(float x, float y, float slope, bool flat, float d1, float d2, float& sigma) {
    float absArctanSlope = (slope != kInf) ? fabs_(fatan(slope)) : 0.5f * float(M_PI);
    float angleM;
    if (x > 0 and y > 0)
      angleM = 0.5f * float(M_PI) - absArctanSlope;
    else if (x < 0 and y > 0)
      angleM = absArctanSlope + 0.5f * float(M_PI);
    else if (x < 0 and y < 0)
      angleM = -(absArctanSlope + 0.5f * float(M_PI));
    else if (x > 0 and y < 0)
      angleM = -(0.5f * float(M_PI) - absArctanSlope);
    else
      angleM = 0;
    float xPrime, yPrime;
    if (!flat) {
      xPrime = x * fcos(angleM) + y * fsin(angleM);
      yPrime = y * fcos(angleM) - x * fsin(angleM);
    } else {
      xPrime = x;
      yPrime = y;
    }
    sigma = 2 * fsqrt((xPrime * d1) * (xPrime * d1) + (yPrime * d2) * (yPrime * d2));
  }

  // Weighted circle regression (SDL/Quintuplet.h:1223-1321).
  LST_HD_BIG float circleRegression(int nPoints,
                                const float* xs,
                                const float* ys,
                                const float* delta1,
                                const float* delta2,
                                const float* slopes,
                                const bool* isFlat,
                                float& g,
                                float& f,
                                float* sigmas,
                                float& chiSquared) {
    float sigmaX1Squared = 0.f, sigmaX2Squared = 0.f, sigmaX1X2 = 0.f, sigmaX1y = 0.f, sigmaX2y = 0.f, sigmaY = 0.f,
          sigmaX1 = 0.f, sigmaX2 = 0.f, sigmaOne = 0.f;
    for (int i = 0; i < nPoints; i++) {
      measurementFrame(xs[i], ys[i], slopes[i], isFlat[i], delta1[i], delta2[i], sigmas[i]);
      sigmaX1Squared += (xs[i] * xs[i]) / (sigmas[i] * sigmas[i]);
      sigmaX2Squared += (ys[i] * ys[i]) / (sigmas[i] * sigmas[i]);
      sigmaX1X2 += (xs[i] * ys[i]) / (sigmas[i] * sigmas[i]);
      sigmaX1y += (xs[i] * (xs[i] * xs[i] + ys[i] * ys[i])) / (sigmas[i] * sigmas[i]);
      sigmaX2y += (ys[i] * (xs[i] * xs[i] + ys[i] * ys[i])) / (sigmas[i] * sigmas[i]);
      sigmaY += (xs[i] * xs[i] + ys[i] * ys[i]) / (sigmas[i] * sigmas[i]);
      sigmaX1 += xs[i] / (sigmas[i] * sigmas[i]);
      sigmaX2 += ys[i] / (sigmas[i] * sigmas[i]);
      sigmaOne += 1.0f / (sigmas[i] * sigmas[i]);
    }
    float denominator = (sigmaX1X2 - sigmaX1 * sigmaX2) * (sigmaX1X2 - sigmaX1 * sigmaX2) -
                        (sigmaX1Squared - sigmaX1 * sigmaX1) * (sigmaX2Squared - sigmaX2 * sigmaX2);
    float twoG = ((sigmaX2y - sigmaX2 * sigmaY) * (sigmaX1X2 - sigmaX1 * sigmaX2) -
                  (sigmaX1y - sigmaX1 * sigmaY) * (sigmaX2Squared - sigmaX2 * sigmaX2)) /
                 denominator;
    float twoF = ((sigmaX1y - sigmaX1 * sigmaY) * (sigmaX1X2 - sigmaX1 * sigmaX2) -
                  (sigmaX2y - sigmaX2 * sigmaY) * (sigmaX1Squared - sigmaX1 * sigmaX1)) /
                 denominator;
    float c = -(sigmaY - twoG * sigmaX1 - twoF * sigmaX2) / sigmaOne;
    g = 0.5f * twoG;
    f = 0.5f * twoF;
    if (g * g + f * f - c < 0) {
      chiSquared = -1;
      return -1;
    }
    float radius = fsqrt(g * g + f * f - c);
    chiSquared = 0.f;
    for (int i = 0; i < nPoints; i++) {
      chiSquared += (xs[i] * xs[i] + ys[i] * ys[i] - twoG * xs[i] - twoF * ys[i] + c) *
                    (xs[i] * xs[i] + ys[i] * ys[i] - twoG * xs[i] - twoF * ys[i] + c) / (sigmas[i] * sigmas[i]);
    }
    return radius;
  }

  // Chi-squared of points against a given circle (SDL/Quintuplet.h:1323-1368,
  // identical to SDL/PixelTriplet.h:370-417 and :2219-2264).
  LST_HD_BIG float circleChi2(int nPoints,
                          const float* xs,
                          const float* ys,
                          const float* delta1,
                          const float* delta2,
                          const float* slopes,
                          const bool* isFlat,
                          float g,
                          float f,
                          float radius) {
    float c = g * g + f * f - radius * radius;
    float chiSquared = 0.f;
    for (int i = 0; i < nPoints; i++) {
      float sigma;
      measurementFrame(xs[i], ys[i], slopes[i], isFlat[i], delta1[i], delta2[i], sigma);
      chiSquared += (xs[i] * xs[i] + ys[i] * ys[i] - 2 * g * xs[i] - 2 * f * ys[i] + c) *
                    (xs[i] * xs[i] + ys[i] * ys[i] - 2 * g * xs[i] - 2 * f * ys[i] + c) / (sigma * sigma);
    }
    return chiSquared;
  }

  // ------------------------------------------------------------- T5 DNN
  // Raw (unstandardised) input features (SDL/NeuralNetwork.h:63-114).
  LST_HD_BIG void t5DnnFeatures(const Modules& m,
                            const MiniDoublets& md,
                            const Segments& s,
                            const Triplets& t,
                            const float* xVec,
                            const float* yVec,
                            const unsigned int* mdIdx,
                            const uint16_t* lm,
                            unsigned int innerT3,
                            float innerRadius,
                            float outerRadius,
                            float bridgeRadius,
                            float* x) {
    short layer2_adjustment = 0;
    if (m.layers[lm[0]] == 1)
      layer2_adjustment = 1;
    unsigned int md_idx_for_t5_eta_phi = s.mdIndices[2 * t.segmentIndices[2 * innerT3 + layer2_adjustment]];
    bool is_endcap[5];
    for (int i = 0; i < 5; ++i)
      is_endcap[i] = (m.subdets[lm[i]] == 4);
    auto hitFeatures = [&](int k, int slot) {
      unsigned int mi = mdIdx[slot];
      x[k + 0] = md.anchorEta[mi];
      x[k + 1] = md.anchorPhi[mi];
      x[k + 2] = md.anchorPos[mi].z;
      x[k + 3] = fsqrt(xVec[slot] * xVec[slot] + yVec[slot] * yVec[slot]);
      x[k + 4] = float(m.layers[lm[slot]] + 6 * is_endcap[slot]);
    };
    x[0] = log10_(2 * k2Rinv1GeVf * innerRadius);
    hitFeatures(1, 0);
    hitFeatures(6, 1);
    hitFeatures(11, 2);
    x[16] = log10_(2 * k2Rinv1GeVf * outerRadius);
    hitFeatures(17, 2);
    hitFeatures(22, 3);
    hitFeatures(27, 4);
    x[32] = log10_((innerRadius + outerRadius) * kMagneticField * 1.602f / (2 * 100 * 5.39f));
    x[33] = md.anchorEta[md_idx_for_t5_eta_phi];
    x[34] = md.anchorPhi[md_idx_for_t5_eta_phi];
    x[35] = log10_(innerRadius);
    x[36] = log10_(bridgeRadius);
    x[37] = log10_(outerRadius);
  }

  // Forward pass, accumulating in the reference's order (SDL/NeuralNetwork.h:116-164).
  template <typename W>
  LST_HD float t5DnnForward(const W& w, const float* x) {
    float h1[32];
#pragma unroll 1
    for (int col = 0; col < 32; ++col) {
      float acc = 0;
      for (int in = 0; in < 38; ++in)
        acc += x[in] * w.w0[in * 32 + col];
      acc += w.b0[col];
      h1[col] = (acc > 0.f) ? acc : 0.f;
    }
    float h2[32];
#pragma unroll 1
    for (int col = 0; col < 32; ++col) {
      float acc = 0;
      for (int in = 0; in < 32; ++in)
        acc += h1[in] * w.w2[in * 32 + col];
      acc += w.b2[col];
      h2[col] = (acc > 0.f) ? acc : 0.f;
    }
    float out = 0;
    for (int in = 0; in < 32; ++in)
      out += h2[in] * w.w4[in];
    out += w.b4[0];
    return fexp(out) / (fexp(out) + 1);
  }

  // ------------------------------------------------------------ T5 driver
  // What the T5 selection sees at the classifier stage (for training and
  // studying the classifier): the 38 DNN inputs, the score of the loaded
  // weights, and the cut-only method's decision on the same candidate.
  struct T5Probe {
    float feat[38];
    float dnnScore;
    bool cutPass;
    bool rzTight;
  };

  struct T5Values {
    float innerRadius, outerRadius, bridgeRadius, regressionG, regressionF, regressionRadius, rzChiSquared, chiSquared,
        nonAnchorChiSquared;
    bool tightCutFlag;
  };

  // A candidate staged for the classifier pass at the end of kT5Eval's
  // block (the event's kT5DnnCap slots are split among the blocks).
  constexpr unsigned int kT5DnnCap = 1u << 14;
  struct T5DnnSlotG {
    T5Values v;
    unsigned int mdIdx[5];
    unsigned int cand;
    uint16_t lm[5];
    uint8_t tight;
  };

  // T5 selection for one (inner T3, outer T3) pair
  // (SDL/Quintuplet.h:2508-2984).  useDnn selects the DNN method
  // (USE_RZCHI2 + USE_T5_DNN) with working point dnnWP (the reference's is
  // kT5DnnWP), otherwise the cut-only method (USE_RZCHI2 + USE_RPHICHI2).
  // With a probe, stops at the classifier stage and fills it instead.
  // State of a candidate at the classifier decision.
  struct T5Stage {
    unsigned int mdIdx[5];
    float xs[5], ys[5];
    bool tight;  // the rz fit's tight flag
    int kind;    // barrel/endcap pattern of the five modules (0: all barrel ... 7)
  };

  // Every test before the classifier decision, and the circle regression.
  // The shared-MD test and the radius tests that open t5SelectPre (the
  // cheapest tests, which most candidates fail); fills the hit coordinates,
  // MD indices and radii the later tests use.
  LST_HD bool t5RadiusStage(const Modules& m,
                            const MiniDoublets& md,
                            const Segments& s,
                            const Triplets& t,
                            const uint16_t* lm,
                            unsigned int innerT3,
                            unsigned int outerT3,
                            T5Values& v,
                            T5Stage& st) {
    unsigned int seg1 = t.segmentIndices[2 * innerT3];
    unsigned int seg2 = t.segmentIndices[2 * innerT3 + 1];
    unsigned int seg3 = t.segmentIndices[2 * outerT3];
    unsigned int seg4 = t.segmentIndices[2 * outerT3 + 1];
    if (s.mdIndices[2 * seg2 + 1] != s.mdIndices[2 * seg3])
      return false;
    unsigned int* mdIdx = st.mdIdx;
    unsigned int mdIdxInit[5] = {s.mdIndices[2 * seg1],
                             s.mdIndices[2 * seg2],
                             s.mdIndices[2 * seg2 + 1],
                             s.mdIndices[2 * seg3 + 1],
                             s.mdIndices[2 * seg4 + 1]};
    for (int i = 0; i < 5; ++i)
      mdIdx[i] = mdIdxInit[i];

    float* xs = st.xs;
    float* ys = st.ys;
    for (int i = 0; i < 5; ++i) {
      xs[i] = md.anchorPos[mdIdx[i]].x;
      ys[i] = md.anchorPos[mdIdx[i]].y;
    }
    float g, f;
    v.outerRadius = t.circleRadius[outerT3];
    v.bridgeRadius = circleFrom3(xs[1], ys[1], xs[2], ys[2], xs[3], ys[3], g, f);
    v.innerRadius = t.circleRadius[innerT3];

    // Every test below is a pure function of the candidate and all must pass,
    // so they run cheapest first: the radius tests of
    // SDL/Quintuplet.h:2740-2906 before the two beta algorithms of :2555-2622
    // and the rz test of :2715-2735.
    const bool pass = (v.innerRadius >= 0.95f * m.ptCut / (2.f * k2Rinv1GeVf));
    if (!pass)
      return false;
    short s1 = m.subdets[lm[0]], s2 = m.subdets[lm[1]], s3 = m.subdets[lm[2]], s4 = m.subdets[lm[3]],
          s5 = m.subdets[lm[4]];
    int kind;
    if (s1 == Barrel and s2 == Barrel and s3 == Barrel and s4 == Barrel and s5 == Barrel)
      kind = 0;
    else if (s1 == Barrel and s2 == Barrel and s3 == Barrel and s4 == Barrel and s5 == Endcap)
      kind = 1;
    else if (s1 == Barrel and s2 == Barrel and s3 == Barrel and s4 == Endcap and s5 == Endcap)
      kind = m.layers[lm[0]] == 1 ? 2 : (m.layers[lm[0]] == 2 ? 3 : 4);
    else if (s1 == Barrel and s2 == Barrel and s3 == Endcap and s4 == Endcap and s5 == Endcap)
      kind = 5;
    else if (s1 == Barrel and s2 == Endcap and s3 == Endcap and s4 == Endcap and s5 == Endcap)
      kind = 6;
    else
      kind = 7;
    st.kind = kind;
    // Radius spreads over the strip ends of 2S endcap hits; only the tests of
    // kinds >= 2 read them (the reference's third, outer spread is unused).
    float innerRadiusMin2S = 0.f, innerRadiusMax2S = 0.f, bridgeRadiusMin2S = 0.f, bridgeRadiusMax2S = 0.f;
    if (kind >= 2) {
      float px[5][3], py[5][3];
      int np[5];
      for (int i = 0; i < 5; ++i) {
        px[i][0] = px[i][1] = px[i][2] = xs[i];
        py[i][0] = py[i][1] = py[i][2] = ys[i];
        np[i] = 1;
        if (m.subdets[lm[i]] == Endcap and m.moduleType[lm[i]] == TwoS) {
          px[i][1] = md.anchorLowEdgeX[mdIdx[i]];
          px[i][2] = md.anchorHighEdgeX[mdIdx[i]];
          py[i][1] = md.anchorLowEdgeY[mdIdx[i]];
          py[i][2] = md.anchorHighEdgeY[mdIdx[i]];
          np[i] = 3;
        }
      }
      if (kind >= 6)
        radiusSpread(px[0], py[0], np[0], px[1], py[1], np[1], px[2], py[2], np[2], innerRadiusMin2S, innerRadiusMax2S);
      radiusSpread(px[1], py[1], np[1], px[2], py[2], np[2], px[3], py[3], np[3], bridgeRadiusMin2S, bridgeRadiusMax2S);
    }
    return matchRadii(
        kind, v.innerRadius, v.bridgeRadius, innerRadiusMin2S, innerRadiusMax2S, bridgeRadiusMin2S, bridgeRadiusMax2S);
  }

  LST_HD bool t5SelectPre(const Modules& m,
                          const MiniDoublets& md,
                          const Segments& s,
                          const Triplets& t,
                          const uint16_t* lm,
                          unsigned int innerT3,
                          unsigned int outerT3,
                          T5Values& v,
                          T5Stage& st) {
    if (!t5RadiusStage(m, md, s, t, lm, innerT3, outerT3, v, st))
      return false;
    const unsigned int* mdIdx = st.mdIdx;
    const float* xs = st.xs;
    const float* ys = st.ys;
    const unsigned int seg1 = t.segmentIndices[2 * innerT3];
    const unsigned int seg3 = t.segmentIndices[2 * outerT3];
    const unsigned int seg4 = t.segmentIndices[2 * outerT3 + 1];
    float g, f;
    T4Input q1{lm[0], lm[1], lm[2], lm[3], seg1, seg3, mdIdx[0], mdIdx[1], mdIdx[2], mdIdx[3]};
    if (!t4Select(m, md, s, q1))
      return false;
    T4Input q2{lm[0], lm[1], lm[3], lm[4], seg1, seg4, mdIdx[0], mdIdx[1], mdIdx[3], mdIdx[4]};
    if (!t4Select(m, md, s, q2))
      return false;

    g = t.circleCenterX[innerT3];
    f = t.circleCenterY[innerT3];
    float inner_pt = 2 * k2Rinv1GeVf * v.innerRadius;
    bool tight = false;
    if (!t5PassRZ(m, md, mdIdx, lm, v.rzChiSquared, inner_pt, v.innerRadius, g, f, tight))
      return false;

    float sigmas[5], delta1[5], delta2[5], slopes[5];
    bool isFlat[5];
    regressionSigmas(m, lm, delta1, delta2, slopes, isFlat, 5, true);
    v.regressionRadius =
        circleRegression(5, xs, ys, delta1, delta2, slopes, isFlat, v.regressionG, v.regressionF, sigmas, v.chiSquared);
    st.tight = tight;
    return true;
  }

  // The chi-squared of the non-anchor hits against the regression circle
  // (SDL/Quintuplet.h:2960-2984), stored with a selected candidate.
  LST_HD void t5NonAnchor(const Modules& m, const MiniDoublets& md, const uint16_t* lm, const unsigned int* mdIdx,
                          T5Values& v) {
    bool isFlat[5];
    float nonAnchorDelta1[5], nonAnchorDelta2[5], nonAnchorSlopes[5];
    float nonAnchorxs[5], nonAnchorys[5];
    for (int i = 0; i < 5; ++i) {
      nonAnchorxs[i] = md.outerX[mdIdx[i]];
      nonAnchorys[i] = md.outerY[mdIdx[i]];
    }
    regressionSigmas(m, lm, nonAnchorDelta1, nonAnchorDelta2, nonAnchorSlopes, isFlat, 5, false);
    v.nonAnchorChiSquared = circleChi2(5,
                                       nonAnchorxs,
                                       nonAnchorys,
                                       nonAnchorDelta1,
                                       nonAnchorDelta2,
                                       nonAnchorSlopes,
                                       isFlat,
                                       v.regressionG,
                                       v.regressionF,
                                       v.regressionRadius);
  }

  // The classifier decision: the DNN with working point dnnWP, or the
  // cut-only method's r-phi chi-squared table.
  template <typename W>
  LST_HD bool t5Classify(const Modules& m,
                         const MiniDoublets& md,
                         const Segments& s,
                         const Triplets& t,
                         const W& dnn,
                         bool useDnn,
                         float dnnWP,
                         const uint16_t* lm,
                         unsigned int innerT3,
                         T5Values& v,
                         T5Stage& st) {
    bool tight = st.tight;
    if (useDnn) {
      float feat[38];
      t5DnnFeatures(m, md, s, t, st.xs, st.ys, st.mdIdx, lm, innerT3, v.innerRadius, v.outerRadius, v.bridgeRadius,
                    feat);
      float inference = t5DnnForward(dnn, feat);
      if (!(inference > dnnWP))
        return false;
      tight = tight and (inference > dnnWP);
    } else {
      if (v.regressionRadius < 5.0f / (2.f * k2Rinv1GeVf)) {
        if (!t5PassRPhiChi2(m, lm, v.chiSquared))
          return false;
      }
    }
    t5NonAnchor(m, md, lm, st.mdIdx, v);
    v.tightCutFlag = tight;
    return true;
  }

  // Full T5 selection (SDL/Quintuplet.h:2508-2984).  useDnn selects the DNN
  // method (USE_RZCHI2 + USE_T5_DNN) with working point dnnWP (the
  // reference's is kT5DnnWP), otherwise the cut-only method (USE_RZCHI2 +
  // USE_RPHICHI2).  With a probe, stops at the classifier stage and fills it
  // instead.
  template <typename W>
  LST_HD bool t5Select(const Modules& m,
                       const MiniDoublets& md,
                       const Segments& s,
                       const Triplets& t,
                       const W& dnn,
                       bool useDnn,
                       float dnnWP,
                       const uint16_t* lm,
                       unsigned int innerT3,
                       unsigned int outerT3,
                       T5Values& v,
                       T5Probe* probe = nullptr) {
    T5Stage st;
    if (!t5SelectPre(m, md, s, t, lm, innerT3, outerT3, v, st))
      return false;
    if (probe) {
      t5DnnFeatures(m, md, s, t, st.xs, st.ys, st.mdIdx, lm, innerT3, v.innerRadius, v.outerRadius, v.bridgeRadius,
                    probe->feat);
      probe->dnnScore = t5DnnForward(dnn, probe->feat);
      probe->cutPass = v.regressionRadius < 5.0f / (2.f * k2Rinv1GeVf) ? t5PassRPhiChi2(m, lm, v.chiSquared) : true;
      probe->rzTight = st.tight;
      return true;
    }
    return t5Classify(m, md, s, t, dnn, useDnn, dnnWP, lm, innerT3, v, st);
  }

  // SDL/Quintuplet.h:150-216 with the eta/phi/pt/score formed in
  // SDL/Quintuplet.h:3072-3079.
  LST_HD void storeT5(const MiniDoublets& md,
                      const Segments& s,
                      Triplets& t,
                      Quintuplets& q,
                      unsigned int innerT3,
                      unsigned int outerT3,
                      const uint16_t* lm,
                      int layer,
                      const T5Values& v,
                      unsigned int idx) {
    short layer2_adjustment = (layer == 1) ? 1 : 0;
    unsigned int etaMD = s.mdIndices[2 * t.segmentIndices[2 * innerT3 + layer2_adjustment]];
    float phi = md.anchorPhi[etaMD];
    float eta = md.anchorEta[etaMD];
    float pt = (v.innerRadius + v.outerRadius) * 3.8f * 1.602f / (2 * 100 * 5.39f);
    float scores = v.chiSquared + v.nonAnchorChiSquared;
    q.tripletIndices[2 * idx] = innerT3;
    q.tripletIndices[2 * idx + 1] = outerT3;
    for (int i = 0; i < 5; ++i)
      q.lowerModuleIndices[5 * idx + i] = lm[i];
    q.innerRadius[idx] = v.innerRadius;
    q.outerRadius[idx] = v.outerRadius;
    q.pt[idx] = pt;
    q.eta[idx] = eta;
    q.phi[idx] = phi;
    q.score_rphisum[idx] = scores;
    q.layer[idx] = static_cast<uint8_t>(layer);
    q.isDup[idx] = 0;
    q.TightCutFlag[idx] = v.tightCutFlag;
    q.partOfPT5[idx] = 0;
    q.regressionRadius[idx] = v.regressionRadius;
    q.regressionG[idx] = v.regressionG;
    q.regressionF[idx] = v.regressionF;
    q.logicalLayers[5 * idx] = t.logicalLayers[3 * innerT3];
    q.logicalLayers[5 * idx + 1] = t.logicalLayers[3 * innerT3 + 1];
    q.logicalLayers[5 * idx + 2] = t.logicalLayers[3 * innerT3 + 2];
    q.logicalLayers[5 * idx + 3] = t.logicalLayers[3 * outerT3 + 1];
    q.logicalLayers[5 * idx + 4] = t.logicalLayers[3 * outerT3 + 2];
    for (int i = 0; i < 6; ++i)
      q.hitIndices[10 * idx + i] = t.hitIndices[6 * innerT3 + i];
    for (int i = 0; i < 4; ++i)
      q.hitIndices[10 * idx + 6 + i] = t.hitIndices[6 * outerT3 + 2 + i];
    q.bridgeRadius[idx] = v.bridgeRadius;
    q.rzChiSquared[idx] = v.rzChiSquared;
    q.chiSquared[idx] = v.chiSquared;
    q.nonAnchorChiSquared[idx] = v.nonAnchorChiSquared;
    t.partOfT5[innerT3] = 1;
    t.partOfT5[outerT3] = 1;
  }

}  // namespace lst
