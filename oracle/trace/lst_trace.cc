// Cut-flip tracer and FP64 re-evaluation of single LST objects (test
// infrastructure; see oracle/tracer.py for the Python side).
//
// The product's cut functions (tracklooper_b200/csrc/lst_*.h) are compiled
// here with `float` replaced by lst_trace::TFloat (tfloat.h), so one object
// can be evaluated again from its hits in three arithmetics: IEEE single
// precision with correctly rounded transcendentals (what the CUDA path and
// the parity oracle compute), IEEE single precision with glibc's float
// transcendentals (what the reference's stock CPU backend computes), and
// double precision.  Every comparison the selection takes is recorded, so
// the Python side can find the cut whose outcome differs between the two
// single-precision evaluations and measure how far its operand lies from its
// threshold.
//
// An object is named by its hits, as oracle/identity.py keys it, and rebuilt
// from them the way the CUDA kernels build it: per-hit values as kHitPrep,
// mini-doublets as kCreateMD + kMDDerived, segments as kCreateLS, triplets
// as kCreateT3, quintuplets as kT5Eval, pixel segments as kPixelIngest,
// pT3 / pT5 as kPixEval (SDL/Hit.h:217-269, MiniDoublet.h:570-992,
// Segment.h:707-885 and :1031-1117, Triplet.h:797-870, Quintuplet.h:2508-3079,
// PixelTriplet.h:826-1124 and :2480-2781).
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "es.h"
#include "tfloat.h"

// ----------------------------------------------------- arithmetic binding
#define LST_MATH_BINDING_PROVIDED 1
namespace lst {
  using lst_trace::TFloat;

  template <typename D, typename F>
  inline TFloat trMath1(TFloat x, D dfn, F ffn) {
    switch (lst_trace::g_mode) {
      case lst_trace::kF32Cr:
        return TFloat::raw(static_cast<double>(static_cast<float>(dfn(x.v))));
      case lst_trace::kF32Glibc:
        return TFloat::raw(static_cast<double>(ffn(static_cast<float>(x.v))));
      default:
        return TFloat::raw(dfn(x.v));
    }
  }
#define LST_TR_MATH(NAME, DF, FF) \
  inline TFloat NAME(TFloat x) { return trMath1(x, [](double a) { return ::DF(a); }, [](float a) { return ::FF(a); }); }
  LST_TR_MATH(fsin, sin, sinf)
  LST_TR_MATH(fcos, cos, cosf)
  LST_TR_MATH(ftan, tan, tanf)
  LST_TR_MATH(fasin, asin, asinf)
  LST_TR_MATH(facos, acos, acosf)
  LST_TR_MATH(fatan, atan, atanf)
  LST_TR_MATH(fsinh, sinh, sinhf)
  LST_TR_MATH(facosh, acosh, acoshf)
  LST_TR_MATH(fexp, exp, expf)
  LST_TR_MATH(flog, log, logf)
#undef LST_TR_MATH
  inline TFloat fatan2(TFloat y, TFloat x) {
    switch (lst_trace::g_mode) {
      case lst_trace::kF32Cr:
        return TFloat::raw(static_cast<double>(static_cast<float>(::atan2(y.v, x.v))));
      case lst_trace::kF32Glibc:
        return TFloat::raw(static_cast<double>(::atan2f(static_cast<float>(y.v), static_cast<float>(x.v))));
      default:
        return TFloat::raw(::atan2(y.v, x.v));
    }
  }
  inline TFloat fabs_(TFloat x) { return TFloat::raw(std::fabs(x.v)); }
  inline double fabs_(double x) { return std::fabs(x); }
  inline TFloat fmin_(TFloat a, TFloat b) { return TFloat::raw(std::fmin(a.v, b.v)); }
  inline TFloat fmax_(TFloat a, TFloat b) { return TFloat::raw(std::fmax(a.v, b.v)); }
  inline TFloat fmin_(TFloat a, float b) { return fmin_(a, TFloat(b)); }
  inline TFloat fmax_(TFloat a, float b) { return fmax_(a, TFloat(b)); }
  inline double fmin_(TFloat a, double b) { return std::fmin(a.v, b); }
  inline double fmax_(TFloat a, double b) { return std::fmax(a.v, b); }
  inline TFloat fsqrt(TFloat x) { return TFloat::raw(lst_trace::rnd(std::sqrt(x.v))); }
  inline double dsqrt(double x) { return std::sqrt(x); }
  inline bool fisnan(TFloat x) { return std::isnan(x.v); }
  inline TFloat fround_(TFloat x) { return TFloat::raw(std::round(x.v)); }
}  // namespace lst

#define float lst_trace::TFloat
#include "lst_pixel.h"
#undef float

using lst_trace::TFloat;

namespace {

  enum Kind : int { kMD = 0, kLS = 1, kT3 = 2, kT5 = 3, kPT3 = 4, kPT5 = 5 };

  // pLS inputs (the 18 arrays of addPixelSegmentToEvent).
  struct PLSIn {
    std::vector<unsigned int> hit[4];
    std::vector<float> dPhiChange, ptIn, ptErr, px, py, pz, eta, etaErr, phi;
    std::vector<int> charge, superbin;
    std::vector<unsigned int> seedIdx;
    std::vector<int8_t> pixelType, isQuad;
  };

  struct Handle {
    lst::EsHost es;
    std::vector<TFloat> drdzs, dxdys, eta, r, geoMapPhi;
    lst::Modules m{};
    lst::T5DnnWeights dnn;  // TFloat weights
    TFloat dnnWP = TFloat(0.f);
    // event inputs
    std::vector<float> x, y, z;
    std::vector<unsigned int> detId, idx;
    std::vector<int> module;  // per hit: module index, -1 unknown
    PLSIn pls;
    std::string err;
  };

  std::vector<TFloat> toT(const std::vector<float>& v) {
    std::vector<TFloat> o(v.size());
    for (size_t i = 0; i < v.size(); ++i)
      o[i] = TFloat(v[i]);
    return o;
  }

  // A scratch event holding one candidate and its constituents.
  struct Scratch {
    static constexpr int kH = 16, kMDn = 8, kLSn = 8, kT3n = 2;
    // hits
    std::vector<TFloat> xs, ys, zs, rts, phis, etas, hex, hey, lex, ley, slope, shXa, shYa, shZn;
    std::vector<uint16_t> hmod;
    std::vector<unsigned int> hidx, hdet;
    std::vector<int> hranges;
    lst::Hits h{};
    std::map<unsigned int, unsigned int> local;
    // mini-doublets
    std::vector<unsigned int> mdA, mdO, mdN, mdTot;
    std::vector<uint16_t> mdMod;
    std::vector<TFloat> mdF[40];
    std::vector<lst::MDPos> mdPos;
    std::vector<lst::MDRec> mdRec;
    lst::MiniDoublets md{};
    // segments
    std::vector<TFloat> lsF[6];
    std::vector<uint16_t> lsIn, lsOut;
    std::vector<unsigned int> lsMD, lsAIn, lsAOut, lsN, lsTot;
    std::vector<unsigned int> plsSeed, plsHits;
    std::vector<int> plsCharge, plsSuperbin;
    std::vector<int8_t> plsType, plsQuad, plsDup;
    std::vector<uint8_t> plsPart;
    std::vector<TFloat> plsF[13];
    lst::Segments s{};
    // triplets
    std::vector<unsigned int> t3Seg, t3N, t3Tot, t3Hits;
    std::vector<uint16_t> t3Mod;
    std::vector<uint8_t> t3LL, t3P5, t3P, t3P3;
    std::vector<TFloat> t3F[4];
    lst::Triplets t{};
    // quintuplets
    std::vector<unsigned int> q5T3, q5N, q5Tot, q5Hits;
    std::vector<uint16_t> q5Mod;
    std::vector<uint8_t> q5Layer, q5Tight, q5Part, q5LL;
    std::vector<int8_t> q5Dup;
    std::vector<TFloat> q5F[13];
    lst::Quintuplets q{};
    // pT3 / pT5
    std::vector<unsigned int> p3Pls, p3T3, p3N, p3Tot, p3Hits;
    std::vector<uint8_t> p3Dup, p3Part, p3LL;
    std::vector<uint16_t> p3Mod;
    std::vector<TFloat> p3F[15];
    lst::PixelTriplets p3{};
    std::vector<unsigned int> p5Pix, p5T5, p5N, p5Tot, p5Hits;
    std::vector<uint8_t> p5Dup, p5LL;
    std::vector<uint16_t> p5Mod;
    std::vector<TFloat> p5F[10];
    lst::PixelQuintuplets p5{};
    std::vector<int> segModIdx;
    lst::Ranges rg{};

    explicit Scratch(unsigned int nModules) {
      auto F = [](std::vector<TFloat>& v, size_t n) {
        v.assign(n, TFloat(0.f));
        return v.data();
      };
      xs.resize(kH); ys.resize(kH); zs.resize(kH); rts.resize(kH); phis.resize(kH); etas.resize(kH);
      hex.resize(kH); hey.resize(kH); lex.resize(kH); ley.resize(kH); slope.resize(kH);
      shXa.resize(kH); shYa.resize(kH); shZn.resize(kH);
      hmod.resize(kH); hidx.resize(kH); hdet.resize(kH); hranges.resize(2 * nModules, -1);
      h.xs = xs.data(); h.ys = ys.data(); h.zs = zs.data(); h.rts = rts.data(); h.phis = phis.data();
      h.etas = etas.data(); h.highEdgeXs = hex.data(); h.highEdgeYs = hey.data(); h.lowEdgeXs = lex.data();
      h.lowEdgeYs = ley.data(); h.moduleIndices = hmod.data(); h.idxs = hidx.data(); h.detid = hdet.data();
      h.hitRanges = hranges.data();

      mdA.resize(kMDn); mdO.resize(kMDn); mdMod.resize(kMDn); mdN.resize(nModules + 1); mdTot.resize(nModules + 1);
      mdPos.resize(kMDn);
      mdRec.resize(kMDn);
      TFloat* f[40];
      for (int i = 0; i < 40; ++i)
        f[i] = F(mdF[i], kMDn);
      md.anchorHitIndices = mdA.data(); md.outerHitIndices = mdO.data(); md.moduleIndices = mdMod.data();
      md.nMDs = mdN.data(); md.totOccupancyMDs = mdTot.data();
      int k = 0;
      md.dphichanges = f[k++]; md.dzs = f[k++]; md.dphis = f[k++]; md.shiftedXs = f[k++]; md.shiftedYs = f[k++];
      md.shiftedZs = f[k++]; md.noShiftedDzs = f[k++]; md.noShiftedDphis = f[k++]; md.noShiftedDphiChanges = f[k++];
      md.anchorX = f[k++]; md.anchorY = f[k++]; md.anchorZ = f[k++]; md.anchorRt = f[k++]; md.anchorPhi = f[k++];
      md.anchorEta = f[k++]; md.anchorHighEdgeX = f[k++]; md.anchorHighEdgeY = f[k++]; md.anchorLowEdgeX = f[k++];
      md.anchorLowEdgeY = f[k++]; md.anchorLowEdgePhi = f[k++]; md.anchorHighEdgePhi = f[k++]; md.outerX = f[k++];
      md.outerY = f[k++]; md.outerZ = f[k++]; md.outerRt = f[k++]; md.outerPhi = f[k++]; md.outerEta = f[k++];
      md.outerHighEdgeX = f[k++]; md.outerHighEdgeY = f[k++]; md.outerLowEdgeX = f[k++]; md.outerLowEdgeY = f[k++];
      md.slope = f[k++]; md.tanSlope = f[k++]; md.slope3 = f[k++];
      md.anchorPos = mdPos.data();
      md.rec = mdRec.data();

      TFloat* g[6];
      for (int i = 0; i < 6; ++i)
        g[i] = F(lsF[i], kLSn);
      s.dPhis = g[0]; s.dPhiMins = g[1]; s.dPhiMaxs = g[2]; s.dPhiChanges = g[3]; s.dPhiChangeMins = g[4];
      s.dPhiChangeMaxs = g[5];
      lsIn.resize(kLSn); lsOut.resize(kLSn); lsMD.resize(2 * kLSn); lsAIn.resize(kLSn); lsAOut.resize(kLSn);
      lsN.resize(nModules + 1); lsTot.resize(nModules + 1);
      s.innerLowerModuleIndices = lsIn.data(); s.outerLowerModuleIndices = lsOut.data(); s.mdIndices = lsMD.data();
      s.innerMiniDoubletAnchorHitIndices = lsAIn.data(); s.outerMiniDoubletAnchorHitIndices = lsAOut.data();
      s.nSegments = lsN.data(); s.totOccupancySegments = lsTot.data();
      plsSeed.resize(1); plsHits.resize(4); plsCharge.resize(1); plsSuperbin.resize(1); plsType.resize(1);
      plsQuad.resize(1); plsDup.resize(1); plsPart.resize(1);
      TFloat* pf[13];
      for (int i = 0; i < 13; ++i)
        pf[i] = F(plsF[i], 1);
      s.seedIdx = plsSeed.data(); s.charge = plsCharge.data(); s.superbin = plsSuperbin.data();
      s.pLSHitsIdxs = plsHits.data(); s.pixelType = plsType.data(); s.isQuad = plsQuad.data(); s.isDup = plsDup.data();
      s.partOfPT5 = plsPart.data();
      s.ptIn = pf[0]; s.ptErr = pf[1]; s.px = pf[2]; s.py = pf[3]; s.pz = pf[4]; s.etaErr = pf[5]; s.eta = pf[6];
      s.phi = pf[7]; s.score = pf[8]; s.circleCenterX = pf[9]; s.circleCenterY = pf[10]; s.circleRadius = pf[11];

      t3Seg.resize(2 * kT3n); t3Mod.resize(3 * kT3n); t3N.resize(nModules); t3Tot.resize(nModules);
      t3LL.resize(3 * kT3n); t3Hits.resize(6 * kT3n); t3P5.resize(kT3n); t3P.resize(kT3n); t3P3.resize(kT3n);
      t.segmentIndices = t3Seg.data(); t.lowerModuleIndices = t3Mod.data(); t.nTriplets = t3N.data();
      t.totOccupancyTriplets = t3Tot.data(); t.logicalLayers = t3LL.data(); t.hitIndices = t3Hits.data();
      t.betaIn = F(t3F[0], kT3n); t.circleRadius = F(t3F[1], kT3n); t.circleCenterX = F(t3F[2], kT3n);
      t.circleCenterY = F(t3F[3], kT3n);
      t.partOfPT5 = t3P5.data(); t.partOfT5 = t3P.data(); t.partOfPT3 = t3P3.data();

      q5T3.resize(2); q5Mod.resize(5); q5N.resize(nModules); q5Tot.resize(nModules); q5Layer.resize(1);
      q5Dup.resize(1); q5Tight.resize(1); q5Part.resize(1); q5LL.resize(5); q5Hits.resize(10);
      TFloat* qf[13];
      for (int i = 0; i < 13; ++i)
        qf[i] = F(q5F[i], 1);
      q.tripletIndices = q5T3.data(); q.lowerModuleIndices = q5Mod.data(); q.nQuintuplets = q5N.data();
      q.totOccupancyQuintuplets = q5Tot.data(); q.innerRadius = qf[0]; q.bridgeRadius = qf[1]; q.outerRadius = qf[2];
      q.pt = qf[3]; q.eta = qf[4]; q.phi = qf[5]; q.score_rphisum = qf[6]; q.layer = q5Layer.data();
      q.isDup = q5Dup.data(); q.TightCutFlag = q5Tight.data(); q.partOfPT5 = q5Part.data();
      q.regressionRadius = qf[7]; q.regressionG = qf[8]; q.regressionF = qf[9]; q.logicalLayers = q5LL.data();
      q.hitIndices = q5Hits.data(); q.rzChiSquared = qf[10]; q.chiSquared = qf[11]; q.nonAnchorChiSquared = qf[12];

      p3Pls.resize(1); p3T3.resize(1); p3N.resize(1); p3Tot.resize(1); p3Dup.resize(1); p3Part.resize(1);
      p3LL.resize(5); p3Hits.resize(10); p3Mod.resize(5);
      TFloat* rf[15];
      for (int i = 0; i < 15; ++i)
        rf[i] = F(p3F[i], 1);
      p3.pixelSegmentIndices = p3Pls.data(); p3.tripletIndices = p3T3.data(); p3.nPixelTriplets = p3N.data();
      p3.totOccupancyPixelTriplets = p3Tot.data(); p3.pixelRadius = rf[0]; p3.tripletRadius = rf[1]; p3.pt = rf[2];
      p3.eta = rf[3]; p3.phi = rf[4]; p3.eta_pix = rf[5]; p3.phi_pix = rf[6]; p3.score = rf[7];
      p3.isDup = p3Dup.data(); p3.partOfPT5 = p3Part.data(); p3.logicalLayers = p3LL.data();
      p3.hitIndices = p3Hits.data(); p3.lowerModuleIndices = p3Mod.data(); p3.centerX = rf[8]; p3.centerY = rf[9];
      p3.pixelRadiusError = rf[10]; p3.rPhiChiSquared = rf[11]; p3.rPhiChiSquaredInwards = rf[12];
      p3.rzChiSquared = rf[13];

      p5Pix.resize(1); p5T5.resize(1); p5N.resize(1); p5Tot.resize(1); p5Dup.resize(1); p5LL.resize(7);
      p5Hits.resize(14); p5Mod.resize(7);
      TFloat* sf[10];
      for (int i = 0; i < 10; ++i)
        sf[i] = F(p5F[i], 1);
      p5.pixelIndices = p5Pix.data(); p5.T5Indices = p5T5.data(); p5.nPixelQuintuplets = p5N.data();
      p5.totOccupancyPixelQuintuplets = p5Tot.data(); p5.isDup = p5Dup.data(); p5.score = sf[0]; p5.eta = sf[1];
      p5.phi = sf[2]; p5.logicalLayers = p5LL.data(); p5.hitIndices = p5Hits.data();
      p5.lowerModuleIndices = p5Mod.data(); p5.pixelRadius = sf[3]; p5.quintupletRadius = sf[4]; p5.centerX = sf[5];
      p5.centerY = sf[6]; p5.rzChiSquared = sf[7]; p5.rPhiChiSquared = sf[8]; p5.rPhiChiSquaredInwards = sf[9];

      segModIdx.assign(nModules + 1, 0);
      rg.segmentModuleIndices = segModIdx.data();
    }
  };

  // The per-hit values of kHitPrep for one hit; returns its local index.
  int prepHit(const Handle& H, Scratch& S, unsigned int g) {
    auto it = S.local.find(g);
    if (it != S.local.end())
      return int(it->second);
    if (g >= H.x.size() || S.local.size() >= size_t(Scratch::kH))
      return -1;
    const int i = int(S.local.size());
    S.local[g] = unsigned(i);
    const lst::Modules& m = H.m;
    TFloat x = TFloat(H.x[g]), y = TFloat(H.y[g]), z = TFloat(H.z[g]);
    S.xs[i] = x;
    S.ys[i] = y;
    S.zs[i] = z;
    S.hidx[i] = H.idx[g];
    S.hdet[i] = H.detId[g];
    TFloat rt = lst::fsqrt(x * x + y * y);
    S.rts[i] = rt;
    S.phis[i] = lst::phiOf(x, y);
    S.etas[i] = ((z > 0) - (z < 0)) * lst::facosh(lst::fsqrt(x * x + y * y + z * z) / rt);
    TFloat hex = TFloat(0.f), hey = TFloat(0.f), lex = TFloat(0.f), ley = TFloat(0.f);
    const int mi = H.module[g];
    if (mi < 0)
      return -1;
    S.hmod[i] = uint16_t(mi);
    S.slope[i] = lst::mdMiniSlope(rt, m.ptCut);
    if (mi != H.es.pixelModuleIndex) {
      const bool isLowerHit = m.isLower[mi];
      const uint16_t lm = isLowerHit ? uint16_t(mi) : m.partnerModuleIndices[mi];
      const bool shifted = m.subdets[lm] == lst::Endcap || (m.subdets[lm] == lst::Barrel && m.sides[lm] != lst::Center);
      if (shifted && lst::shiftMovesLower(m, lm) == isLowerHit) {
        TFloat xa, ya, zn;
        lst::shiftStripPrep(m, lm, x, y, z, rt, xa, ya, zn);
        S.shXa[i] = xa;
        S.shYa[i] = ya;
        S.shZn[i] = zn;
      }
    }
    if (m.subdets[mi] == lst::Endcap && m.moduleType[mi] == lst::TwoS) {
      const int f = m.geoMapIndex[mi];
      if (f >= 0) {
        TFloat phi = m.geoMapPhi[f];
        TFloat cos_phi = lst::fcos(phi);
        hex = x + 2.5f * cos_phi;
        lex = x - 2.5f * cos_phi;
        TFloat sin_phi = lst::fsin(phi);
        hey = y + 2.5f * sin_phi;
        ley = y - 2.5f * sin_phi;
      }
    }
    S.hex[i] = hex;
    S.hey[i] = hey;
    S.lex[i] = lex;
    S.ley[i] = ley;
    return i;
  }

  // A mini-doublet of two outer-tracker hits given as (anchor, outer), as
  // kCreateMD selects and stores it; returns its local index or -1.
  int buildMD(const Handle& H, Scratch& S, int& nMD, unsigned int a, unsigned int o, bool& pass) {
    const lst::Modules& m = H.m;
    int la = prepHit(H, S, a), lo = prepHit(H, S, o);
    if (la < 0 || lo < 0 || nMD >= Scratch::kMDn)
      return -1;
    uint16_t ma = S.hmod[la], mo = S.hmod[lo];
    const bool aLower = m.isLower[ma];
    const uint16_t lm = aLower ? ma : mo;
    const int lower = aLower ? la : lo, upper = aLower ? lo : la;
    lst::MDHitPre pre{S.slope.data(), S.shXa.data(), S.shYa.data(), S.shZn.data()};
    lst::MDValues v;
    pass = lst::mdSelect(m, lm, S.xs[lower], S.ys[lower], S.zs[lower], S.rts[lower], S.xs[upper], S.ys[upper],
                         S.zs[upper], S.rts[upper], S.phis[lower], S.phis[upper], pre, unsigned(lower), unsigned(upper), v);
    const int idx = nMD++;
    lst::storeMD(m, S.h, S.md, unsigned(lower), unsigned(upper), lm, v, unsigned(idx));
    lst::storeMDDerived(S.md, unsigned(idx), H.m.ptCut);
    return idx;
  }

  int buildLS(const Handle& H, Scratch& S, int& nLS, int md0, int md1, bool& pass) {
    lst::LSValues v;
    const uint16_t inLM = S.mdMod[md0], outLM = S.mdMod[md1];
    pass = lst::lsSelect(H.m, S.md, inLM, outLM, unsigned(md0), unsigned(md1), v);
    const int idx = nLS++;
    lst::storeLS(S.s, S.md, unsigned(md0), unsigned(md1), inLM, outLM, v, unsigned(idx));
    return idx;
  }

  int buildT3(const Handle& H, Scratch& S, int& nT3, int ls0, int ls1, bool& pass) {
    const uint16_t lm1 = S.mdMod[S.lsMD[2 * ls0]], lm2 = S.mdMod[S.lsMD[2 * ls0 + 1]], lm3 = S.mdMod[S.lsMD[2 * ls1 + 1]];
    lst::T3Values v{TFloat(0.f), TFloat(0.f), TFloat(0.f), TFloat(0.f)};
    pass = lst::t3Select(H.m, S.md, S.s, lm1, lm2, lm3, unsigned(ls0), unsigned(ls1), v);
    const int idx = nT3++;
    lst::storeT3(H.m, S.md, S.s, S.t, unsigned(ls0), unsigned(ls1), lm1, lm2, lm3, v, unsigned(idx));
    return idx;
  }

  // Builds the outer-tracker chain of nHits/2 mini-doublets given as (anchor,
  // outer) hit pairs: MDs, the segments between consecutive MDs, and (for 6
  // or 10 hits) the triplets; the object being traced is built last, with
  // the trace recording.  fail collects a bit per constituent that fails.
  struct Chain {
    int md[5] = {-1, -1, -1, -1, -1};
    int ls[4] = {-1, -1, -1, -1};
    int t3[2] = {-1, -1};
    int nMD = 0, nLS = 0, nT3 = 0;
  };

  bool buildChain(const Handle& H, Scratch& S, const unsigned int* hits, int nPairs, Chain& c, unsigned int& fail,
                  int lastLevel, std::vector<lst_trace::Rec>* trace, bool& lastPass) {
    // lastLevel: 0 MD, 1 LS, 2 T3 -- the level whose (single) object is traced
    auto traced = [&](bool on) { lst_trace::g_trace = on ? trace : nullptr; };
    for (int i = 0; i < nPairs; ++i) {
      bool p;
      traced(lastLevel == 0);
      c.md[i] = buildMD(H, S, c.nMD, hits[2 * i], hits[2 * i + 1], p);
      traced(false);
      if (c.md[i] < 0)
        return false;
      if (lastLevel == 0)
        lastPass = p;
      else if (!p)
        fail |= 1u << i;
    }
    if (lastLevel == 0)
      return true;
    for (int i = 0; i + 1 < nPairs; ++i) {
      if (nPairs == 5 && i == 2) {
        // a quintuplet's triplets are (MD0, MD1, MD2) and (MD2, MD3, MD4)
      }
      bool p;
      traced(lastLevel == 1);
      c.ls[i] = buildLS(H, S, c.nLS, c.md[i], c.md[i + 1], p);
      traced(false);
      if (lastLevel == 1)
        lastPass = p;
      else if (!p)
        fail |= 1u << (8 + i);
    }
    if (lastLevel == 1)
      return true;
    const int nT3 = nPairs == 3 ? 1 : 2;
    for (int k = 0; k < nT3; ++k) {
      bool p;
      traced(lastLevel == 2);
      c.t3[k] = buildT3(H, S, c.nT3, c.ls[2 * k], c.ls[2 * k + 1], p);
      traced(false);
      if (lastLevel == 2)
        lastPass = p;
      else if (!p)
        fail |= 1u << (16 + k);
    }
    return true;
  }

  // The pLS with array index p, as kPixelIngest stores it (segment index 4,
  // mini-doublets 5 and 6 of the scratch event).
  constexpr int kPlsSeg = 4, kPlsMD = 5;
  bool buildPLS(const Handle& H, Scratch& S, unsigned int p) {
    const PLSIn& in = H.pls;
    if (p >= in.ptIn.size())
      return false;
    int lh[4];
    for (int k = 0; k < 4; ++k) {
      lh[k] = prepHit(H, S, in.hit[k][p]);
      if (lh[k] < 0)
        return false;
    }
    S.s.ptIn[0] = TFloat(in.ptIn[p]);
    S.s.ptErr[0] = TFloat(in.ptErr[p]);
    S.s.px[0] = TFloat(in.px[p]);
    S.s.py[0] = TFloat(in.py[p]);
    S.s.pz[0] = TFloat(in.pz[p]);
    S.s.eta[0] = TFloat(in.eta[p]);
    S.s.etaErr[0] = TFloat(in.etaErr[p]);
    S.s.phi[0] = TFloat(in.phi[p]);
    S.s.charge[0] = in.charge[p];
    S.s.superbin[0] = in.superbin[p];
    S.s.seedIdx[0] = in.seedIdx[p];
    S.s.pixelType[0] = in.pixelType[p];
    S.s.isQuad[0] = in.isQuad[p];
    const uint16_t pix = H.es.pixelModuleIndex;
    S.rg.segmentModuleIndices[pix] = kPlsSeg;
    lst::storePixelSegment(H.m, S.h, S.md, S.s, pix, kPlsMD, kPlsSeg, 0, unsigned(lh[0]), unsigned(lh[1]),
                           unsigned(lh[2]), unsigned(lh[3]), TFloat(in.dPhiChange[p]));
    lst::storeMDDerived(S.md, kPlsMD, H.m.ptCut);
    lst::storeMDDerived(S.md, kPlsMD + 1, H.m.ptCut);
    return true;
  }

  void put(double* out, int cap, int& n, TFloat v) {
    if (n < cap)
      out[n] = v.v;
    ++n;
  }

}  // namespace

extern "C" {

void* lsttr_create(const char* geometry_dir, const float* dnn_weights, float dnn_wp) {
  Handle* H = new Handle();
  H->err = lst::loadEsHost(geometry_dir, H->es);
  if (!H->err.empty()) {
    delete H;
    return nullptr;
  }
  const lst::EsHost& e = H->es;
  H->drdzs = toT(e.drdzs);
  H->dxdys = toT(e.dxdys);
  H->eta = toT(e.eta);
  H->r = toT(e.r);
  H->geoMapPhi = toT(e.geoMapPhi);
  lst::Modules& m = H->m;
  m.detIds = e.detIds.data();
  m.moduleMap = e.moduleMap.data();
  m.mapdetId = e.mapdetId.data();
  m.mapIdx = e.mapIdx.data();
  m.nConnectedModules = e.nConnectedModules.data();
  m.drdzs = H->drdzs.data();
  m.dxdys = H->dxdys.data();
  m.partnerModuleIndices = e.partnerModuleIndices.data();
  m.layers = e.layers.data();
  m.rings = e.rings.data();
  m.modules = e.modules.data();
  m.rods = e.rods.data();
  m.subdets = e.subdets.data();
  m.sides = e.sides.data();
  m.eta = H->eta.data();
  m.r = H->r.data();
  m.isInverted = e.isInverted.data();
  m.isLower = e.isLower.data();
  m.isAnchor = e.isAnchor.data();
  m.moduleType = e.moduleType.data();
  m.moduleLayerType = e.moduleLayerType.data();
  m.sdlLayers = e.sdlLayers.data();
  m.connectedPixels = e.connectedPixels.data();
  m.geoMapDetId = e.geoMapDetId.data();
  m.geoMapPhi = H->geoMapPhi.data();
  m.geoMapIndex = e.geoMapIndex.data();
  m.nEndCapMap = unsigned(e.geoMapDetId.size());
  m.nModules = e.nModules;
  m.nLowerModules = e.nLowerModules;
  m.ptCut = TFloat(e.ptCut);
  TFloat* w = reinterpret_cast<TFloat*>(&H->dnn);
  static_assert(sizeof(lst::T5DnnWeights) == lst::kT5DnnParams * sizeof(TFloat), "TFloat weight layout");
  for (int i = 0; i < lst::kT5DnnParams; ++i)
    w[i] = TFloat(dnn_weights[i]);
  H->dnnWP = TFloat(dnn_wp);
  return H;
}

void lsttr_destroy(void* h) { delete static_cast<Handle*>(h); }

int lsttr_set_hits(void* h, unsigned int n, const float* x, const float* y, const float* z, const unsigned int* detId,
                   const unsigned int* idx) {
  Handle* H = static_cast<Handle*>(h);
  H->x.assign(x, x + n);
  H->y.assign(y, y + n);
  H->z.assign(z, z + n);
  H->detId.assign(detId, detId + n);
  H->idx.assign(idx, idx + n);
  H->module.assign(n, -1);
  const auto& md = H->es.mapdetId;
  for (unsigned int i = 0; i < n; ++i) {
    auto it = std::lower_bound(md.begin(), md.end(), detId[i]);
    if (it != md.end() && *it == detId[i])
      H->module[i] = H->es.mapIdx[size_t(it - md.begin())];
  }
  return 0;
}

int lsttr_set_pls(void* h, unsigned int n, const unsigned int* h0, const unsigned int* h1, const unsigned int* h2,
                  const unsigned int* h3, const float* dPhiChange, const float* ptIn, const float* ptErr,
                  const float* px, const float* py, const float* pz, const float* eta, const float* etaErr,
                  const float* phi, const int* charge, const unsigned int* seedIdx, const int* superbin,
                  const int8_t* pixelType, const int8_t* isQuad) {
  PLSIn& p = static_cast<Handle*>(h)->pls;
  p.hit[0].assign(h0, h0 + n);
  p.hit[1].assign(h1, h1 + n);
  p.hit[2].assign(h2, h2 + n);
  p.hit[3].assign(h3, h3 + n);
  p.dPhiChange.assign(dPhiChange, dPhiChange + n);
  p.ptIn.assign(ptIn, ptIn + n);
  p.ptErr.assign(ptErr, ptErr + n);
  p.px.assign(px, px + n);
  p.py.assign(py, py + n);
  p.pz.assign(pz, pz + n);
  p.eta.assign(eta, eta + n);
  p.etaErr.assign(etaErr, etaErr + n);
  p.phi.assign(phi, phi + n);
  p.charge.assign(charge, charge + n);
  p.seedIdx.assign(seedIdx, seedIdx + n);
  p.superbin.assign(superbin, superbin + n);
  p.pixelType.assign(pixelType, pixelType + n);
  p.isQuad.assign(isQuad, isQuad + n);
  return 0;
}

// Evaluates one object in the given arithmetic (lst_trace::Mode).  key: the
// hits of an MD (2), LS (4), T3 (6) or T5 (10) as (anchor, outer) pairs; for
// pT3 / pT5 the pLS array index followed by the object's 10 / 14 hits (4
// pixel hits, then the triplet's / quintuplet's).  Returns 1 if the object
// passes, 0 if not, -1 on a malformed key.  values receives the object's
// stored floats (order in oracle/tracer.py), trace the comparisons of its own
// selection, *fail a bit per constituent that fails in this arithmetic.
int lsttr_eval(void* h, int mode, int kind, int use_dnn, const unsigned int* key, int key_len, double* values,
               int values_cap, int* n_values, lst_trace::Rec* trace, int trace_cap, int* n_trace,
               unsigned int* fail) {
  Handle* H = static_cast<Handle*>(h);
  lst_trace::g_mode = mode;
  std::vector<lst_trace::Rec> tr;
  Scratch S(H->es.nModules);
  Chain c;
  unsigned int f = 0;
  bool pass = false;
  int nv = 0;
  static const int kHitsOf[6] = {2, 4, 6, 10, 10, 14};
  const int pixel = (kind == kPT3 || kind == kPT5) ? 1 : 0;
  if (kind < 0 || kind > kPT5 || key_len != kHitsOf[kind] + pixel)
    return -1;
  const unsigned int* hits = key + pixel + (pixel ? 4 : 0);
  const int nPairs = (kHitsOf[kind] - (pixel ? 4 : 0)) / 2;
  auto finish = [&](int rc) {
    lst_trace::g_trace = nullptr;
    if (n_trace)
      *n_trace = int(tr.size());
    if (trace)
      for (int i = 0; i < int(tr.size()) && i < trace_cap; ++i)
        trace[i] = tr[size_t(i)];
    if (n_values)
      *n_values = nv;
    if (fail)
      *fail = f;
    return rc;
  };
  if (kind <= kT3) {
    if (!buildChain(*H, S, hits, nPairs, c, f, kind, &tr, pass))
      return finish(-1);
    if (kind == kMD) {
      const int i = c.md[0];
      for (auto* arr : {S.md.dzs, S.md.dphis, S.md.dphichanges, S.md.noShiftedDzs, S.md.noShiftedDphis,
                        S.md.noShiftedDphiChanges, S.md.shiftedXs, S.md.shiftedYs, S.md.shiftedZs})
        put(values, values_cap, nv, arr[i]);
    } else if (kind == kLS) {
      const int i = c.ls[0];
      for (auto* arr : {S.s.dPhis, S.s.dPhiMins, S.s.dPhiMaxs, S.s.dPhiChanges, S.s.dPhiChangeMins,
                        S.s.dPhiChangeMaxs})
        put(values, values_cap, nv, arr[i]);
    } else {
      const int i = c.t3[0];
      for (auto* arr : {S.t.betaIn, S.t.circleRadius, S.t.circleCenterX, S.t.circleCenterY})
        put(values, values_cap, nv, arr[i]);
    }
    return finish(pass ? 1 : 0);
  }
  // quintuplet chain (T5, and the T5 of a pT5) or triplet chain (pT3)
  bool dummy = false;
  if (!buildChain(*H, S, hits, nPairs, c, f, 3, &tr, dummy))
    return finish(-1);
  uint16_t lm[5] = {0, 0, 0, 0, 0};
  if (nPairs == 5) {
    lm[0] = S.t.lowerModuleIndices[0];
    lm[1] = S.t.lowerModuleIndices[1];
    lm[2] = S.t.lowerModuleIndices[2];
    lm[3] = S.t.lowerModuleIndices[4];
    lm[4] = S.t.lowerModuleIndices[5];
    lst::T5Values v{};
    lst_trace::g_trace = kind == kT5 ? &tr : nullptr;
    const bool ok = lst::t5Select(H->m, S.md, S.s, S.t, H->dnn, use_dnn != 0, H->dnnWP, lm, 0u, 1u, v);
    lst_trace::g_trace = nullptr;
    lst::storeT5(S.md, S.s, S.t, S.q, 0u, 1u, lm, H->m.layers[lm[0]], v, 0u);
    // the DNN score of the candidate (not stored by the reference)
    TFloat score = TFloat(-1.f);
    {
      lst::T5Values v2{};
      lst::T5Stage st;
      if (lst::t5SelectPre(H->m, S.md, S.s, S.t, lm, 0u, 1u, v2, st)) {
        TFloat feat[38];
        lst::t5DnnFeatures(H->m, S.md, S.s, S.t, st.xs, st.ys, st.mdIdx, lm, 0u, v2.innerRadius, v2.outerRadius,
                           v2.bridgeRadius, feat);
        score = lst::t5DnnForward(H->dnn, feat);
      }
    }
    if (kind == kT5) {
      const lst::Quintuplets& q = S.q;
      for (auto* arr : {q.innerRadius, q.bridgeRadius, q.outerRadius, q.pt, q.eta, q.phi, q.score_rphisum,
                        q.regressionRadius, q.regressionG, q.regressionF, q.rzChiSquared, q.chiSquared,
                        q.nonAnchorChiSquared})
        put(values, values_cap, nv, arr[0]);
      put(values, values_cap, nv, score);
      put(values, values_cap, nv, TFloat(double(q.TightCutFlag[0])));
      return finish(ok ? 1 : 0);
    }
    if (!ok)
      f |= 1u << 24;
  }
  // pixel objects
  if (!buildPLS(*H, S, key[0]))
    return finish(-1);
  const unsigned int plsIndex = kPlsSeg;
  if (kind == kPT3) {
    lst::PT3Values v{};
    lst_trace::g_trace = &tr;
    const bool ok = lst::pt3Select(H->m, S.rg, S.md, S.s, S.t, plsIndex, 0u, true, v);
    lst_trace::g_trace = nullptr;
    const short adj = H->m.layers[S.t.lowerModuleIndices[0]] == 1 ? 1 : 0;
    lst::storePT3(H->m, S.md, S.s, S.t, S.p3, plsIndex, 0u, 0u, adj, v, 0u);
    const lst::PixelTriplets& p = S.p3;
    for (auto* arr : {p.pixelRadius, p.pixelRadiusError, p.tripletRadius, p.pt, p.eta, p.phi, p.eta_pix, p.phi_pix,
                      p.score, p.rPhiChiSquared, p.rPhiChiSquaredInwards, p.rzChiSquared})
      put(values, values_cap, nv, arr[0]);
    return finish(ok ? 1 : 0);
  }
  lst::PT5Values v{};
  lst_trace::g_trace = &tr;
  const bool ok = lst::pt5Select(H->m, S.rg, S.md, S.s, S.t, S.q, plsIndex, 0u, 0u, v);
  lst_trace::g_trace = nullptr;
  lst::storePT5(S.md, S.s, S.t, S.q, S.p5, plsIndex, 0u, 0u, v, 0u);
  const lst::PixelQuintuplets& p = S.p5;
  for (auto* arr : {p.pixelRadius, p.quintupletRadius, p.score, p.eta, p.phi, p.centerX, p.centerY, p.rzChiSquared,
                    p.rPhiChiSquared, p.rPhiChiSquaredInwards})
    put(values, values_cap, nv, arr[0]);
  return finish(ok ? 1 : 0);
}

// Code address -> offset from the library's load base (for addr2line).
unsigned long long lsttr_site_offset(const void* site) {
  Dl_info info;
  if (!dladdr(site, &info) || !info.dli_fbase)
    return 0;
  return static_cast<unsigned long long>(static_cast<const char*>(site) - static_cast<const char*>(info.dli_fbase));
}

}  // extern "C"
