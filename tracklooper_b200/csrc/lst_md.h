// Mini-doublet (MD) selection: a pair of hits on the two sensors of one
// outer-tracker module.  Cut arithmetic follows SDL/MiniDoublet.h:193-892.
#pragma once

#include "lst_core.h"

namespace lst {

  // SDL/Constants.h:124-129 (double literals rounded to float, as there)
  LST_HD float miniMulsPtScaleBarrel(unsigned int i) {
    switch (i) {
      case 0: return static_cast<float>(0.0052);
      case 1: return static_cast<float>(0.0038);
      case 2: return static_cast<float>(0.0034);
      case 3: return static_cast<float>(0.0034);
      case 4: return static_cast<float>(0.0032);
      default: return static_cast<float>(0.0034);
    }
  }
  LST_HD float miniMulsPtScaleEndcap(unsigned int) { return static_cast<float>(0.006); }
  LST_HD float miniRminMeanBarrel(unsigned int i) {
    switch (i) {
      case 0: return static_cast<float>(25.007152356);
      case 1: return static_cast<float>(37.2186993757);
      case 2: return static_cast<float>(52.3104270826);
      case 3: return static_cast<float>(68.6658656666);
      case 4: return static_cast<float>(85.9770373007);
      default: return static_cast<float>(108.301772384);
    }
  }
  LST_HD float miniRminMeanEndcap(unsigned int i) {
    switch (i) {
      case 0: return static_cast<float>(130.992832231);
      case 1: return static_cast<float>(154.813883559);
      case 2: return static_cast<float>(185.352604327);
      case 3: return static_cast<float>(221.635123002);
      default: return static_cast<float>(265.022076742);
    }
  }

  // Tilted barrel modules with the smaller sensor spacing (SDL/MiniDoublet.h:268-286).
  LST_HD bool isTighterTilted(short subdet, short layer, short side, short rod) {
    return (subdet == Barrel) && (((side != Center) && (layer == 3)) ||
                                  ((side == NegZ) && (((layer == 2) && (rod > 5)) || ((layer == 1) && (rod > 9)))) ||
                                  ((side == PosZ) && (((layer == 2) && (rod < 8)) || ((layer == 1) && (rod < 4)))));
  }

  // Separation of the two sensors of a module (SDL/MiniDoublet.h:288-337).
  LST_HD float moduleGap(short layer, short ring, short subdet, short side, short rod) {
    unsigned int iL = layer - 1;
    unsigned int iR = ring - 1;
    if (subdet == Barrel && side == Center) {
      switch (iL) {
        case 0: return 0.26f;
        case 1: return 0.16f;
        case 2: return 0.16f;
        default: return 0.18f;
      }
    } else if (isTighterTilted(subdet, layer, side, rod)) {
      return 0.26f;
    } else if (subdet == Endcap) {
      unsigned int nWide = (iL <= 1) ? 10u : ((iL <= 3) ? 8u : 9u);
      return iR < nWide ? 0.4f : 0.18f;
    }
    return 0.4f;
  }
  LST_HD float moduleGap(const Modules& m, unsigned int i) {
    return moduleGap(m.layers[i], m.rings[i], m.subdets[i], m.sides[i], m.rods[i]);
  }

  // dPhi acceptance of a mini-doublet (SDL/MiniDoublet.h:340-402).
  // The slope term of mdDPhiThreshold, a function of the hit's rt alone
  // (computed once per hit by kHitPrep).
  LST_HD float mdMiniSlope(float rt, float ptCut) { return fasin(fmin_(rt * k2Rinv1GeVf / ptCut, kSinAlphaMax)); }

  LST_HD float mdDPhiThresholdFromSlope(const Modules& m, float miniSlope, uint16_t mi, float dPhi = 0, float dz = 0) {
    unsigned int iL = m.layers[mi] - 1;
    const bool barrel = m.subdets[mi] == Barrel;
    const float rLayNominal = barrel ? miniRminMeanBarrel(iL) : miniRminMeanEndcap(iL);
    const float miniPVoff = 0.1f / rLayNominal;
    const float miniMuls =
        barrel ? miniMulsPtScaleBarrel(iL) * 3.f / m.ptCut : miniMulsPtScaleEndcap(iL) * 3.f / m.ptCut;
    const bool isTilted = barrel and m.sides[mi] != Center;
    float drdz;
    if (isTilted) {
      if (m.moduleType[mi] == PS and m.moduleLayerType[mi] == Strip)
        drdz = m.drdzs[mi];
      else
        drdz = m.drdzs[m.partnerModuleIndices[mi]];
    } else {
      drdz = 0;
    }
    const float miniTilt =
        isTilted ? 0.5f * kPixelPSZpitch * drdz / fsqrt(1.f + drdz * drdz) / moduleGap(m, mi) : 0;
    const float miniLum = fabs_(dPhi * kDeltaZLum / dz);
    if (barrel and m.sides[mi] == Center)
      return miniSlope + fsqrt(miniMuls * miniMuls + miniPVoff * miniPVoff);
    else if (barrel)
      return miniSlope + fsqrt(miniMuls * miniMuls + miniPVoff * miniPVoff + miniTilt * miniTilt * miniSlope * miniSlope);
    return miniSlope + fsqrt(miniMuls * miniMuls + miniPVoff * miniPVoff + miniLum * miniLum);
  }

  LST_HD float mdDPhiThreshold(const Modules& m, float rt, uint16_t mi, float dPhi = 0, float dz = 0) {
    return mdDPhiThresholdFromSlope(m, mdMiniSlope(rt, m.ptCut), mi, dPhi, dz);
  }

  // Moves the strip hit along the strip so that it lines up with the
  // interaction point and the pixel hit (SDL/MiniDoublet.h:404-568).
  // shiftStripHit (SDL/MiniDoublet.h:110-191) moves one hit of the pair (p)
  // along the strip direction onto the other sensor's plane and projects it
  // next to the other hit (o).  Which hit is p depends only on the lower
  // module lm: true = the lower hit.
  LST_HD bool shiftMovesLower(const Modules& m, uint16_t lm) {
    if (m.moduleType[lm] == PS)
      return m.subdets[lm] == Barrel ? m.moduleLayerType[lm] != Pixel : m.moduleLayerType[lm] == Pixel;
    return true;
  }

  // The part of shiftStripHit that depends on p alone: the moved point before
  // the projection (xa, ya) and the moved z (computed once per hit by kHitPrep).
  LST_HD void shiftStripPrep(const Modules& m, uint16_t lm, float xp, float yp, float zp, float rtp, float& xa, float& ya,
                             float& zn) {
    const float slope = m.dxdys[lm];
    const float drdz_ = m.drdzs[lm];
    const bool isEndcap = m.subdets[lm] == Endcap;
    float angleA = fabs_(fatan(rtp / zp));
    float angleB = isEndcap ? float(M_PI) / 2.f : fatan(drdz_);
    float moduleSeparation = moduleGap(m, lm);
    if (m.moduleType[lm] == PS and m.moduleLayerType[lm] != Pixel)
      moduleSeparation *= -1;
    float drprime = (moduleSeparation / fsin(angleA + angleB)) * fsin(angleA);
    float absArctanSlope = (slope != kInf) ? fabs_(fatan(slope)) : float(M_PI) / 2.f;
    float angleM;
    if (xp > 0 and yp > 0)
      angleM = absArctanSlope;
    else if (xp > 0 and yp < 0)
      angleM = float(M_PI) - absArctanSlope;
    else if (xp < 0 and yp < 0)
      angleM = float(M_PI) + absArctanSlope;
    else
      angleM = 2.f * float(M_PI) - absArctanSlope;
    float drprime_x = drprime * fsin(angleM);
    float drprime_y = drprime * fcos(angleM);
    xa = xp + drprime_x;
    ya = yp + drprime_y;
    float absdzprime = fabs_(moduleSeparation / fsin(angleA + angleB) * fcos(angleA));
    float abszn;
    if (m.moduleLayerType[lm] == Pixel)
      abszn = fabs_(zp) + absdzprime;
    else
      abszn = fabs_(zp) - absdzprime;
    zn = abszn * ((zp > 0) ? 1 : -1);
  }

  // The projection next to the other hit (xo, yo) that completes shiftStripHit.
  LST_HD void shiftStripFinish(const Modules& m, uint16_t lm, float xa, float ya, float xo, float yo, float& xn,
                               float& yn) {
    const float slope = m.dxdys[lm];
    if (slope == kInf) {
      xn = xa;
      yn = yo;
    } else if (slope == 0) {
      xn = xo;
      yn = ya;
    } else {
      xn = (slope * xa + (1.f / slope) * xo - ya + yo) / (slope + (1.f / slope));
      yn = (xn - xa) * slope + ya;
    }
  }

  // Per-hit values of the mini-doublet cuts computed once per hit: the slope
  // term of the dphi threshold and, for the hit that shiftStripHit moves, its
  // moved point (xa, ya) and z.  Arrays indexed by hit.
  struct MDHitPre {
    const float* miniSlope;
    const float* shiftXa;
    const float* shiftYa;
    const float* shiftZn;
  };

  LST_HD void shiftStripHit(const Modules& m,
                            uint16_t lm,
                            const MDHitPre& pre,
                            unsigned int lowerIdx,
                            unsigned int upperIdx,
                            float xLower,
                            float yLower,
                            float xUpper,
                            float yUpper,
                            float& xn,
                            float& yn,
                            float& zn) {
    const bool fromLower = shiftMovesLower(m, lm);
    const unsigned int p = fromLower ? lowerIdx : upperIdx;
    const float xo = fromLower ? xUpper : xLower, yo = fromLower ? yUpper : yLower;
    zn = pre.shiftZn[p];
    shiftStripFinish(m, lm, pre.shiftXa[p], pre.shiftYa[p], xo, yo, xn, yn);
  }

  // The derived per-MD values of MiniDoublets (slope, tanSlope, slope3).
  // Also fills the mini-doublet's record of segment-cut inputs (MDRec).
  LST_HD void storeMDDerived(MiniDoublets& md, unsigned int idx, float ptCut) {
    const float rt = md.anchorRt[idx];
    const float slope = fasin(fmin_(rt * k2Rinv1GeVf / ptCut, kSinAlphaMax));
    const float tanSlope = ftan(slope);
    md.slope[idx] = slope;
    md.tanSlope[idx] = tanSlope;
    md.slope3[idx] = fasin(fmin_(rt * k2Rinv1GeVf / 3.0f, kSinAlphaMax));
    const MDPos p = md.anchorPos[idx];
    md.rec[idx] = MDRec{p.x, p.y, p.z, p.rt, md.anchorPhi[idx], slope, tanSlope, md.dphichanges[idx],
                        md.dphis[idx], md.dzs[idx], md.anchorHighEdgePhi[idx], md.anchorLowEdgePhi[idx]};
  }

  struct MDValues {
    float dz, dphi, dphichange, shiftedX, shiftedY, shiftedZ, noShiftedDz, noShiftedDphi, noShiftedDphiChange;
  };

  // Barrel mini-doublet (SDL/MiniDoublet.h:645-777).
  LST_HD_BIG bool mdBarrel(const Modules& m,
                       uint16_t lm,
                       float xLower,
                       float yLower,
                       float zLower,
                       float rtLower,
                       float xUpper,
                       float yUpper,
                       float zUpper,
                       float rtUpper,
                       float phiLower,
                       float phiUpper,
                       const MDHitPre& pre,
                       unsigned int lowerIdx,
                       unsigned int upperIdx,
                       MDValues& v) {
    v.dz = zLower - zUpper;
    const float dzCut = m.moduleType[lm] == PS ? 2.f : 10.f;
    const float sign = ((v.dz > 0) - (v.dz < 0)) * ((zLower > 0) - (zLower < 0));
    const float invertedcrossercut = (fabs_(v.dz) > 2) * sign;
    if (!((fabs_(v.dz) < dzCut) && (invertedcrossercut <= 0)))
      return false;

    const bool lowerIsPixel = m.moduleLayerType[lm] == Pixel;
    float miniCut = mdDPhiThresholdFromSlope(m, pre.miniSlope[lowerIsPixel ? lowerIdx : upperIdx], lm);

    float shiftedRt = 0;
    const bool tilted = m.sides[lm] != Center;
    if (tilted) {
      float xn, yn, zn;
      shiftStripHit(m, lm, pre, lowerIdx, upperIdx, xLower, yLower, xUpper, yUpper, xn, yn, zn);
      v.shiftedX = xn;
      v.shiftedY = yn;
      shiftedRt = fsqrt(xn * xn + yn * yn);
      if (lowerIsPixel) {
        v.shiftedZ = zUpper;
        v.dphi = phiMpiPi(phiOf(v.shiftedX, v.shiftedY) - phiLower);
      } else {
        v.shiftedZ = zLower;
        v.dphi = phiMpiPi(phiUpper - phiOf(v.shiftedX, v.shiftedY));
      }
      v.noShiftedDphi = phiMpiPi(phiUpper - phiLower);
    } else {
      v.shiftedX = 0;
      v.shiftedY = 0;
      v.shiftedZ = 0;
      v.dphi = phiMpiPi(phiUpper - phiLower);
      v.noShiftedDphi = v.dphi;
    }
    if (!(fabs_(v.dphi) < miniCut))
      return false;

    if (tilted) {
      if (!lowerIsPixel) {
        v.dphichange = (rtLower < shiftedRt) ? deltaPhiChangeFrom(phiLower, xLower, yLower, v.shiftedX, v.shiftedY)
                                             : deltaPhiChange(v.shiftedX, v.shiftedY, xLower, yLower);
      } else {
        v.dphichange = (shiftedRt < rtUpper) ? deltaPhiChange(v.shiftedX, v.shiftedY, xUpper, yUpper)
                                             : deltaPhiChangeFrom(phiUpper, xUpper, yUpper, v.shiftedX, v.shiftedY);
      }
      v.noShiftedDphiChange = rtLower < rtUpper ? deltaPhiChangeFrom(phiLower, xLower, yLower, xUpper, yUpper)
                                                : deltaPhiChangeFrom(phiUpper, xUpper, yUpper, xLower, yLower);
    } else {
      v.dphichange = deltaPhiChangeFrom(phiLower, xLower, yLower, xUpper, yUpper);
      v.noShiftedDphiChange = v.dphichange;
    }
    v.noShiftedDz = 0;
    return fabs_(v.dphichange) < miniCut;
  }

  // Endcap mini-doublet (SDL/MiniDoublet.h:779-892).  The stored "dz" of an
  // endcap mini-doublet is the transverse-radius difference.
  LST_HD_BIG bool mdEndcap(const Modules& m,
                       uint16_t lm,
                       float xLower,
                       float yLower,
                       float zLower,
                       float rtLower,
                       float xUpper,
                       float yUpper,
                       float zUpper,
                       float rtUpper,
                       float phiLower,
                       float phiUpper,
                       const MDHitPre& pre,
                       unsigned int lowerIdx,
                       unsigned int upperIdx,
                       MDValues& v) {
    float dz = zLower - zUpper;
    const float dzCut = 1.f;
    if (!(fabs_(dz) < dzCut))
      return false;
    const float drtCut = m.moduleType[lm] == PS ? 2.f : 10.f;
    v.dz = rtLower - rtUpper;
    if (!(fabs_(v.dz) < drtCut))
      return false;

    float xn, yn, zn;
    shiftStripHit(m, lm, pre, lowerIdx, upperIdx, xLower, yLower, xUpper, yUpper, xn, yn, zn);
    const bool isPS = m.moduleType[lm] == PS;
    const bool lowerIsPixel = m.moduleLayerType[lm] == Pixel;
    v.shiftedX = xn;
    v.shiftedY = yn;
    if (isPS) {
      if (lowerIsPixel) {
        v.shiftedZ = zUpper;
        v.dphi = phiMpiPi(phiOf(v.shiftedX, v.shiftedY) - phiLower);
      } else {
        v.shiftedZ = zLower;
        v.dphi = phiMpiPi(phiUpper - phiOf(v.shiftedX, v.shiftedY));
      }
    } else {
      v.shiftedZ = zUpper;
      v.dphi = phiMpiPi(phiOf(xn, yn) - phiLower);
    }
    v.noShiftedDphi = phiMpiPi(phiUpper - phiLower);

    if (isPS)
      dz = lowerIsPixel ? zLower - zn : zUpper - zn;

    float miniCut = mdDPhiThresholdFromSlope(m, pre.miniSlope[lowerIsPixel ? lowerIdx : upperIdx], lm, v.dphi, dz);
    if (!(fabs_(v.dphi) < miniCut))
      return false;

    float dzFrac = fabs_(dz) / fabs_(zLower);
    v.dphichange = v.dphi / dzFrac * (1.f + dzFrac);
    v.noShiftedDphiChange = v.noShiftedDphi / dzFrac * (1.f + dzFrac);
    v.noShiftedDz = 0;
    return fabs_(v.dphichange) < miniCut;
  }

  // phiLower / phiUpper are the hits' stored phi (hits.phis, phi() of the same
  // coordinates), used wherever the reference takes deltaPhi of a hit itself.
  LST_HD bool mdSelect(const Modules& m,
                       uint16_t lm,
                       float xLower,
                       float yLower,
                       float zLower,
                       float rtLower,
                       float xUpper,
                       float yUpper,
                       float zUpper,
                       float rtUpper,
                       float phiLower,
                       float phiUpper,
                       const MDHitPre& pre,
                       unsigned int lowerIdx,
                       unsigned int upperIdx,
                       MDValues& v) {
    if (m.subdets[lm] == Barrel)
      return mdBarrel(m, lm, xLower, yLower, zLower, rtLower, xUpper, yUpper, zUpper, rtUpper, phiLower, phiUpper, pre,
                      lowerIdx, upperIdx, v);
    return mdEndcap(m, lm, xLower, yLower, zLower, rtLower, xUpper, yUpper, zUpper, rtUpper, phiLower, phiUpper, pre,
                    lowerIdx, upperIdx, v);
  }

  // Writes a mini-doublet record (SDL/MiniDoublet.h:193-266).  On PS modules
  // whose lower sensor is the strip sensor the anchor is the upper (pixel) hit.
  LST_HD void storeMD(const Modules& m,
                      const Hits& h,
                      MiniDoublets& md,
                      unsigned int lowerHitIdx,
                      unsigned int upperHitIdx,
                      uint16_t lowerModuleIdx,
                      const MDValues& v,
                      unsigned int idx) {
    md.moduleIndices[idx] = lowerModuleIdx;
    unsigned int anchor, outer;
    if (m.moduleType[lowerModuleIdx] == PS and m.moduleLayerType[lowerModuleIdx] == Strip) {
      anchor = upperHitIdx;
      outer = lowerHitIdx;
    } else {
      anchor = lowerHitIdx;
      outer = upperHitIdx;
    }
    md.anchorHitIndices[idx] = anchor;
    md.outerHitIndices[idx] = outer;
    md.dphichanges[idx] = v.dphichange;
    md.dphis[idx] = v.dphi;
    md.dzs[idx] = v.dz;
    md.shiftedXs[idx] = v.shiftedX;
    md.shiftedYs[idx] = v.shiftedY;
    md.shiftedZs[idx] = v.shiftedZ;
    md.noShiftedDzs[idx] = v.noShiftedDz;
    md.noShiftedDphis[idx] = v.noShiftedDphi;
    md.noShiftedDphiChanges[idx] = v.noShiftedDphiChange;

    md.anchorX[idx] = h.xs[anchor];
    md.anchorY[idx] = h.ys[anchor];
    md.anchorZ[idx] = h.zs[anchor];
    md.anchorRt[idx] = h.rts[anchor];
    md.anchorPos[idx] = MDPos{h.xs[anchor], h.ys[anchor], h.zs[anchor], h.rts[anchor]};
    md.anchorPhi[idx] = h.phis[anchor];
    md.anchorEta[idx] = h.etas[anchor];
    float hex = h.highEdgeXs[anchor], hey = h.highEdgeYs[anchor];
    float lex = h.lowEdgeXs[anchor], ley = h.lowEdgeYs[anchor];
    md.anchorHighEdgeX[idx] = hex;
    md.anchorHighEdgeY[idx] = hey;
    md.anchorLowEdgeX[idx] = lex;
    md.anchorLowEdgeY[idx] = ley;
    md.anchorHighEdgePhi[idx] = fatan2(hey, hex);
    md.anchorLowEdgePhi[idx] = fatan2(ley, lex);

    md.outerX[idx] = h.xs[outer];
    md.outerY[idx] = h.ys[outer];
    md.outerZ[idx] = h.zs[outer];
    md.outerRt[idx] = h.rts[outer];
    md.outerPhi[idx] = h.phis[outer];
    md.outerEta[idx] = h.etas[outer];
    md.outerHighEdgeX[idx] = h.highEdgeXs[outer];
    md.outerHighEdgeY[idx] = h.highEdgeYs[outer];
    md.outerLowEdgeX[idx] = h.lowEdgeXs[outer];
    md.outerLowEdgeY[idx] = h.lowEdgeYs[outer];
  }

  // Per-module mini-doublet capacity from the (category, |eta|) occupancy table
  // (SDL/MiniDoublet.h:1019-1067).
  LST_HD int occupancyCategory(short layers, short subdets, short rings) {
    if (layers <= 3 && subdets == 5)
      return 0;
    if (layers >= 4 && subdets == 5)
      return 1;
    if (layers <= 2 && subdets == 4 && rings >= 11)
      return 2;
    if (layers >= 3 && subdets == 4 && rings >= 8)
      return 2;
    if (layers <= 2 && subdets == 4 && rings <= 10)
      return 3;
    if (layers >= 3 && subdets == 4 && rings <= 7)
      return 3;
    return -1;
  }
  LST_HD int occupancyEtaBin(float absEta) {
    if (absEta < 0.75)
      return 0;
    if (absEta > 0.75 && absEta < 1.5)
      return 1;
    if (absEta > 1.5 && absEta < 2.25)
      return 2;
    if (absEta > 2.25 && absEta < 3)
      return 3;
    return -1;
  }
  LST_HD int mdOccupancy(int category, int etaBin) {
    if (category == 0 && etaBin == 0) return 49;
    if (category == 0 && etaBin == 1) return 42;
    if (category == 0 && etaBin == 2) return 37;
    if (category == 0 && etaBin == 3) return 41;
    if (category == 1) return 100;
    if (category == 2 && etaBin == 1) return 16;
    if (category == 2 && etaBin == 2) return 19;
    if (category == 3 && etaBin == 1) return 14;
    if (category == 3 && etaBin == 2) return 20;
    if (category == 3 && etaBin == 3) return 25;
    return 0;
  }
  // SDL/Segment.h:954-994
  LST_HD int lsOccupancy(int category, int etaBin) {
    if (category == 0 && etaBin == 0) return 572;
    if (category == 0 && etaBin == 1) return 300;
    if (category == 0 && etaBin == 2) return 183;
    if (category == 0 && etaBin == 3) return 62;
    if (category == 1 && etaBin == 0) return 191;
    if (category == 1 && etaBin == 1) return 128;
    if (category == 2 && etaBin == 1) return 107;
    if (category == 2 && etaBin == 2) return 102;
    if (category == 3 && etaBin == 1) return 64;
    if (category == 3 && etaBin == 2) return 79;
    if (category == 3 && etaBin == 3) return 85;
    return 0;
  }
  // SDL/Triplet.h:1049-1089
  LST_HD int t3Occupancy(int category, int etaBin) {
    if (category == 0 && etaBin == 0) return 543;
    if (category == 0 && etaBin == 1) return 235;
    if (category == 0 && etaBin == 2) return 88;
    if (category == 0 && etaBin == 3) return 46;
    if (category == 1 && etaBin == 0) return 755;
    if (category == 1 && etaBin == 1) return 347;
    if (category == 2 && etaBin == 1) return 0;
    if (category == 2 && etaBin == 2) return 0;
    if (category == 3 && etaBin == 1) return 38;
    if (category == 3 && etaBin == 2) return 46;
    if (category == 3 && etaBin == 3) return 39;
    return 0;
  }
  // SDL/Quintuplet.h:3179-3198
  LST_HD int t5Occupancy(int category, int etaBin) {
    if (category == 0 && etaBin == 0) return 336;
    if (category == 0 && etaBin == 1) return 414;
    if (category == 0 && etaBin == 2) return 231;
    if (category == 0 && etaBin == 3) return 146;
    if (category == 3 && etaBin == 1) return 0;
    if (category == 3 && etaBin == 2) return 191;
    if (category == 3 && etaBin == 3) return 106;
    return 0;
  }

}  // namespace lst
