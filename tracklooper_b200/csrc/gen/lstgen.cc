// Seeded synthetic event generator for the LST object-building chain.
//
// Produces, per event, exactly the inputs SDL::Event::addHitToEvent and
// SDL::Event::addPixelSegmentToEvent consume (SDL/Event.h:113-137): outer-tracker
// hits (x, y, z, detId, index) followed by the pixel-seed pseudo-hits, and the 18
// pixel-line-segment (pLS) arrays, built with the conventions of the reference's
// standalone input preparation (code/core/trkCore.cc:574-842).
//
// Physics model (stated assumptions, not reference data):
//  * charged particles follow ideal helices in a uniform Bz = 3.8 T field
//    (helix convention of code/core/SDLMath.h:57-99), no material effects;
//  * each sensor of the OT800_IT615 geometry is a flat rectangle centred on its
//    centroid (data/.../sensor_centroids.bin).  Barrel flat sensors face the
//    beam line, tilted barrel sensors lie along dr/dz = drdz of
//    tilted_barrel_orientation.bin, endcap sensors lie in z = const with strips
//    along the radial direction through the centroid.  Nominal active areas
//    (the geometry files carry none): PS 4.7 cm (strip axis) x 9.8 cm, 2S
//    10.0 cm x 9.1 cm;
//  * one hit per crossed sensor on the first outgoing half turn.  Along the
//    strip axis the coordinate is the centre of the crossed strip row (PS strip
//    2.35 cm rows, 2S 5.0 cm rows) or of the macro-pixel (0.15 cm, PS pixel);
//    across it a Gaussian smear of 30 um (strip sensors) or 10 um (PS pixel);
//  * pixel seeds come from the true helix: momentum and impact parameters at the
//    point of closest approach to the beam line, and the state at the last seed
//    hit taken at a nominal inner-tracker radius of 16 cm (or where |z| reaches
//    30 cm, whichever comes first); a quadruplet with probability 0.75, else a
//    triplet; duplicate seeds sharing 3 pixel hits with the first (half of the
//    seeded tracks, and half of the quadruplets once more) and fake seeds (half
//    as many as seeded tracks, see generate()) bring a PU200 event to about
//    1.4e4 pLS after the reference's pLS pT cut;
//  * noise: extra hits, 1% of the signal hit count, uniformly over OT sensors.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <string>
#include <vector>

namespace {

  constexpr double kPi = 3.14159265358979323846;
  constexpr double kBField = 3.8;
  constexpr double kR1GeV = 1.0 / (2.99792458e-3 * kBField);  // cm per GeV of pT

  // ---------------------------------------------------------------- RNG
  // xoshiro256** seeded by splitmix64 (both public-domain algorithms by
  // S. Vigna / D. Blackman).
  struct Rng {
    uint64_t s[4];
    static uint64_t splitmix(uint64_t& x) {
      uint64_t z = (x += 0x9e3779b97f4a7c15ULL);
      z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
      z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
      return z ^ (z >> 31);
    }
    explicit Rng(uint64_t seed) {
      for (auto& w : s)
        w = splitmix(seed);
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
      uint64_t r = rotl(s[1] * 5, 7) * 9;
      uint64_t t = s[1] << 17;
      s[2] ^= s[0];
      s[3] ^= s[1];
      s[1] ^= s[2];
      s[0] ^= s[3];
      s[2] ^= t;
      s[3] = rotl(s[3], 45);
      return r;
    }
    double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
    double uniform(double a, double b) { return a + (b - a) * uniform(); }
    double normal() {
      double u1 = uniform();
      double u2 = uniform();
      if (u1 < 1e-300)
        u1 = 1e-300;
      return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * kPi * u2);
    }
    int poisson(double mean) {
      // Knuth's product method in chunks of 30 to avoid underflow for large means.
      int k = 0;
      double remaining = mean;
      while (remaining > 0) {
        double m = std::min(remaining, 30.0);
        remaining -= m;
        double L = std::exp(-m), p = 1.0;
        int kk = -1;
        do {
          ++kk;
          p *= uniform();
        } while (p > L);
        k += kk;
      }
      return k;
    }
  };

  // ---------------------------------------------------------------- geometry
  struct Sensor {
    uint32_t detId;
    int type;  // 23 PS pixel, 24 PS strip, 25 2S
    int subdet, layer, side;
    double c[3], n[3], u[3], v[3];
    double halfU, halfV, rowU, sigmaV;
  };

  struct Shell {
    // A group of sensors at (nearly) the same radius (barrel) or |z| (endcap).
    bool barrel;
    double pos;  // mean radius (barrel) or signed z (endcap)
    int nPhi, nW;
    double wMin, wStep;  // second binning coordinate: z (barrel) or r (endcap)
    std::vector<std::vector<int>> bins;
  };

  struct Geometry {
    std::vector<Sensor> sensors;
    std::vector<Shell> shells;
    std::map<uint32_t, int> byDetId;
  };

  template <typename T>
  bool readRecords(const std::string& path, std::vector<T>& out) {
    std::ifstream f(path, std::ios::binary);
    if (!f)
      return false;
    T rec;
    while (f.read(reinterpret_cast<char*>(&rec), sizeof(T)))
      out.push_back(rec);
    return true;
  }

#pragma pack(push, 1)
  struct CentroidRec {
    uint32_t detId;
    float x, y, z;
    int32_t type;
  };
  struct OrientRec {
    uint32_t detId;
    float a, b;
  };
#pragma pack(pop)

  bool buildGeometry(const std::string& dir, Geometry& g) {
    std::vector<CentroidRec> cents;
    std::vector<OrientRec> tilted, endcap;
    if (!readRecords(dir + "/sensor_centroids.bin", cents) || cents.empty())
      return false;
    readRecords(dir + "/tilted_barrel_orientation.bin", tilted);
    readRecords(dir + "/endcap_orientation.bin", endcap);
    std::map<uint32_t, float> drdz;
    for (auto& t : tilted)
      drdz[t.detId] = t.a;

    for (auto& cr : cents) {
      Sensor s{};
      s.detId = cr.detId;
      s.type = cr.type;
      s.subdet = (cr.detId >> 25) & 7;
      s.side = s.subdet == 4 ? (cr.detId >> 23) & 3 : (cr.detId >> 18) & 3;
      s.layer = s.subdet == 4 ? (cr.detId >> 18) & 7 : (cr.detId >> 20) & 7;
      s.c[0] = cr.x;
      s.c[1] = cr.y;
      s.c[2] = cr.z;
      double phi = std::atan2(s.c[1], s.c[0]);
      double rh[3] = {std::cos(phi), std::sin(phi), 0.0};
      double ph[3] = {-std::sin(phi), std::cos(phi), 0.0};
      if (s.subdet == 5) {
        double k = 0.0;
        if (s.side != 3) {
          auto it = drdz.find(cr.detId);
          if (it == drdz.end())
            it = drdz.find(cr.detId ^ 1u);
          if (it != drdz.end())
            k = it->second;
        }
        double nrm = std::sqrt(1.0 + k * k);
        for (int i = 0; i < 3; ++i) {
          s.u[i] = (k * rh[i] + (i == 2 ? 1.0 : 0.0)) / nrm;
          s.n[i] = (rh[i] - (i == 2 ? k : 0.0)) / nrm;
          s.v[i] = ph[i];
        }
      } else {
        for (int i = 0; i < 3; ++i) {
          s.u[i] = rh[i];
          s.v[i] = ph[i];
          s.n[i] = (i == 2) ? 1.0 : 0.0;
        }
      }
      if (s.type == 25) {
        s.halfU = 5.0;
        s.halfV = 4.55;
        s.rowU = 5.0;
        s.sigmaV = 30e-4;
      } else if (s.type == 24) {
        s.halfU = 2.35;
        s.halfV = 4.9;
        s.rowU = 2.35;
        s.sigmaV = 30e-4;
      } else {
        s.halfU = 2.35;
        s.halfV = 4.9;
        s.rowU = 0.15;
        s.sigmaV = 10e-4;
      }
      g.byDetId[s.detId] = static_cast<int>(g.sensors.size());
      g.sensors.push_back(s);
    }

    // Group sensors into shells: per (subdet, layer, side-class), cluster by
    // radius (barrel) or z (endcap) with gaps larger than 0.8 cm.
    std::map<std::tuple<int, int, int>, std::vector<int>> groups;
    for (int i = 0; i < (int)g.sensors.size(); ++i) {
      auto& s = g.sensors[i];
      int cls = s.subdet == 5 ? (s.side == 3 ? 0 : s.side) : s.side;
      groups[{s.subdet, s.layer, cls}].push_back(i);
    }
    for (auto& [key, ids] : groups) {
      bool barrel = std::get<0>(key) == 5;
      auto coord = [&](int i) {
        auto& s = g.sensors[i];
        return barrel ? std::hypot(s.c[0], s.c[1]) : s.c[2];
      };
      std::sort(ids.begin(), ids.end(), [&](int a, int b) { return coord(a) < coord(b); });
      size_t start = 0;
      for (size_t k = 1; k <= ids.size(); ++k) {
        if (k < ids.size() && coord(ids[k]) - coord(ids[k - 1]) < 0.8)
          continue;
        Shell sh;
        sh.barrel = barrel;
        double sum = 0;
        double wmin = 1e30, wmax = -1e30;
        for (size_t j = start; j < k; ++j) {
          auto& s = g.sensors[ids[j]];
          sum += coord(ids[j]);
          double w = barrel ? s.c[2] : std::hypot(s.c[0], s.c[1]);
          wmin = std::min(wmin, w);
          wmax = std::max(wmax, w);
        }
        sh.pos = sum / double(k - start);
        sh.nPhi = 256;
        sh.wStep = 4.0;
        sh.wMin = wmin - 8.0;
        sh.nW = int((wmax + 8.0 - sh.wMin) / sh.wStep) + 1;
        sh.bins.assign(size_t(sh.nPhi) * sh.nW, {});
        for (size_t j = start; j < k; ++j) {
          auto& s = g.sensors[ids[j]];
          double phi = std::atan2(s.c[1], s.c[0]);
          double w = barrel ? s.c[2] : std::hypot(s.c[0], s.c[1]);
          int ip = int((phi + kPi) / (2 * kPi) * sh.nPhi) % sh.nPhi;
          int iw = int((w - sh.wMin) / sh.wStep);
          sh.bins[size_t(ip) * sh.nW + iw].push_back(ids[j]);
        }
        g.shells.push_back(std::move(sh));
        start = k;
      }
    }
    return true;
  }

  // ---------------------------------------------------------------- helix
  struct Helix {
    double vx, vy, vz, R, phi0, tanL, q;
    double cx, cy;
    Helix(double pt, double eta, double phi, double x, double y, double z, double charge)
        : vx(x), vy(y), vz(z), R(pt * kR1GeV), phi0(phi), tanL(std::sinh(eta)), q(charge) {
      cx = vx + q * R * std::sin(phi0);
      cy = vy - q * R * std::cos(phi0);
    }
    void at(double t, double* p) const {
      p[0] = cx - q * R * std::sin(phi0 - q * t);
      p[1] = cy + q * R * std::cos(phi0 - q * t);
      p[2] = vz + R * tanL * t;
    }
    void dir(double t, double* d) const {  // dP/dt
      d[0] = R * std::cos(phi0 - q * t);
      d[1] = R * std::sin(phi0 - q * t);
      d[2] = R * tanL;
    }
    // Momentum direction angle in the transverse plane at parameter t.
    double phiAt(double t) const { return phi0 - q * t; }
  };

  struct SimHit {
    double lu, lv;  // local coordinates on the sensor plane (strip axis, precise axis)
    int sensor;
    int particle;
  };

  // First crossing (t in (0, pi)) of the helix with the transverse radius rs.
  bool crossRadius(const Helix& h, double rs, double& t) {
    double pt2R = 2.0 * h.R;
    if (rs >= pt2R * 0.999)
      return false;
    t = 2.0 * std::asin(rs / pt2R);
    for (int it = 0; it < 6; ++it) {
      double p[3], d[3];
      h.at(t, p);
      h.dir(t, d);
      double f = p[0] * p[0] + p[1] * p[1] - rs * rs;
      double fp = 2.0 * (p[0] * d[0] + p[1] * d[1]);
      if (std::fabs(fp) < 1e-12)
        break;
      t -= f / fp;
    }
    return t > 0 && t < kPi;
  }

  // Exact crossing of the helix with the plane of sensor s near parameter t0.
  bool crossSensor(const Helix& h, const Sensor& s, double t0, double& t, double* p, double& lu, double& lv) {
    t = t0;
    for (int it = 0; it < 8; ++it) {
      double d[3];
      h.at(t, p);
      h.dir(t, d);
      double f = (p[0] - s.c[0]) * s.n[0] + (p[1] - s.c[1]) * s.n[1] + (p[2] - s.c[2]) * s.n[2];
      double fp = d[0] * s.n[0] + d[1] * s.n[1] + d[2] * s.n[2];
      if (std::fabs(fp) < 1e-12)
        return false;
      double dt = f / fp;
      t -= dt;
      if (std::fabs(dt) < 1e-10)
        break;
    }
    if (!(t > 0 && t < kPi))
      return false;
    h.at(t, p);
    double r[3] = {p[0] - s.c[0], p[1] - s.c[1], p[2] - s.c[2]};
    lu = r[0] * s.u[0] + r[1] * s.u[1] + r[2] * s.u[2];
    lv = r[0] * s.v[0] + r[1] * s.v[1] + r[2] * s.v[2];
    return std::fabs(lu) <= s.halfU && std::fabs(lv) <= s.halfV;
  }

  void propagate(const Geometry& g, const Helix& h, int particle, std::vector<SimHit>& out) {
    for (auto const& sh : g.shells) {
      double t0;
      if (sh.barrel) {
        if (!crossRadius(h, sh.pos, t0))
          continue;
      } else {
        if (h.tanL == 0.0)
          continue;
        t0 = (sh.pos - h.vz) / (h.R * h.tanL);
        if (!(t0 > 0 && t0 < kPi))
          continue;
      }
      double p[3];
      h.at(t0, p);
      double phi = std::atan2(p[1], p[0]);
      double w = sh.barrel ? p[2] : std::hypot(p[0], p[1]);
      int ip = int((phi + kPi) / (2 * kPi) * sh.nPhi) % sh.nPhi;
      int iw = int(std::floor((w - sh.wMin) / sh.wStep));
      for (int dp = -2; dp <= 2; ++dp) {
        int jp = (ip + dp + sh.nPhi) % sh.nPhi;
        for (int dw = -3; dw <= 3; ++dw) {
          int jw = iw + dw;
          if (jw < 0 || jw >= sh.nW)
            continue;
          for (int si : sh.bins[size_t(jp) * sh.nW + jw]) {
            double t, q[3], lu, lv;
            if (crossSensor(h, g.sensors[si], t0, t, q, lu, lv))
              out.push_back(SimHit{lu, lv, si, particle});
          }
        }
      }
    }
  }

  // ---------------------------------------------------------------- event
  struct Particle {
    double pt, eta, phi, q, vx, vy, vz;
  };

  struct Event {
    // hits: OT hits first (grouped by sensor detId), then pixel pseudo-hits
    std::vector<float> x, y, z;
    std::vector<uint32_t> detId, idx;
    std::vector<int> simIdx;
    uint32_t nOT = 0;
    // pLS
    std::vector<uint32_t> h0, h1, h2, h3, seedIdx;
    std::vector<float> dPhiChange, ptIn, ptErr, px, py, pz, eta, etaErr, phi;
    std::vector<int> charge, superbin, plsSim;
    std::vector<int8_t> pixelType;
    std::vector<char> isQuad;
    std::vector<Particle> particles;
    // The same seeds before conversion, in the CMSSW layout LST::run takes
    // (SDL/LST.h:32-52), every seed including those the pT cut drops; see_f
    // holds the 13 float arrays see_px .. see_stateTrajGlbPz in that order.
    std::vector<float> see_f[13];
    std::vector<int> see_q, see_sim;
    std::vector<uint32_t> see_hitOff{0};
    std::vector<int> see_hitIdx;
  };

  struct Config {
    int id;
    double pileup;         // mean number of pileup vertices (Poisson)
    bool pileupRandom;     // per-event mean drawn U(140, 250)
    double displacedFrac;  // fraction of particles with displaced production
  };

  double sampleHardPt(Rng& r) {
    // pT in [1, 200] GeV with density proportional to pT^-2.
    double u = r.uniform();
    return 1.0 / (1.0 - u * (1.0 - 1.0 / 200.0));
  }

  void makeParticles(const Config& cfg, Rng& r, std::vector<Particle>& ps) {
    if (cfg.id == 1) {
      Particle p;
      p.pt = r.uniform(0.5, 50.0);
      p.eta = r.uniform(-2.4, 2.4);
      p.phi = r.uniform(-kPi, kPi);
      p.q = r.uniform() < 0.5 ? -1.0 : 1.0;
      p.vx = 15e-4 * r.normal();
      p.vy = 15e-4 * r.normal();
      p.vz = 3.5 * r.normal();
      ps.push_back(p);
      return;
    }
    // Hard process: ~20 charged tracks from the primary vertex.
    double pvz = 3.5 * r.normal();
    double pvx = 15e-4 * r.normal(), pvy = 15e-4 * r.normal();
    int nHard = r.poisson(20.0);
    for (int i = 0; i < nHard; ++i) {
      Particle p;
      p.pt = sampleHardPt(r);
      p.eta = r.uniform(-3.0, 3.0);
      p.phi = r.uniform(-kPi, kPi);
      p.q = r.uniform() < 0.5 ? -1.0 : 1.0;
      p.vx = pvx;
      p.vy = pvy;
      p.vz = pvz;
      ps.push_back(p);
    }
    double mean = cfg.pileupRandom ? r.uniform(140.0, 250.0) : cfg.pileup;
    int nVtx = r.poisson(mean);
    for (int v = 0; v < nVtx; ++v) {
      double vz = 3.5 * r.normal();
      double vx = 15e-4 * r.normal(), vy = 15e-4 * r.normal();
      int n = r.poisson(60.0);
      for (int i = 0; i < n; ++i) {
        Particle p;
        p.pt = 0.4 - 0.6 * std::log(1.0 - r.uniform());  // exp(-pT/0.6) truncated below 0.4
        p.eta = r.uniform(-3.0, 3.0);
        p.phi = r.uniform(-kPi, kPi);
        p.q = r.uniform() < 0.5 ? -1.0 : 1.0;
        p.vx = vx;
        p.vy = vy;
        p.vz = vz;
        if (cfg.displacedFrac > 0 && r.uniform() < cfg.displacedFrac) {
          double rr = r.uniform(0.0, 10.0), ph = r.uniform(-kPi, kPi);
          p.vx += rr * std::cos(ph);
          p.vy += rr * std::sin(ph);
        }
        ps.push_back(p);
      }
    }
  }

  float f32(double v) { return static_cast<float>(v); }

  // Seed parameters at the point of closest approach (PCA) to the beam line and
  // at the last seed hit, converted like code/core/trkCore.cc:679-806.
  void addSeed(Event& ev,
               const Helix& h,
               const Particle& p,
               int particle,
               Rng& r,
               uint32_t pixBase,
               int nHits,
               bool shifted) {
    // Momentum at the production point (prompt tracks: the PCA).
    double pxPCA = p.pt * std::cos(p.phi), pyPCA = p.pt * std::sin(p.phi), pzPCA = p.pt * std::sinh(p.eta);
    double relPt = 0.01 * (1.0 + std::fabs(p.eta) / 2.0);
    double scale = 1.0 + relPt * r.normal();
    double dphi = 1e-3 * r.normal();
    double cphi = std::cos(dphi), sphi = std::sin(dphi);
    double spx = scale * (pxPCA * cphi - pyPCA * sphi), spy = scale * (pxPCA * sphi + pyPCA * cphi);
    double spz = scale * pzPCA * (1.0 + 1e-3 * r.normal());
    // Transverse/longitudinal impact parameters relative to the beam line.
    double dxy = (p.vx * std::sin(p.phi) - p.vy * std::cos(p.phi)) + 20e-4 * r.normal();
    double dz = p.vz + 50e-4 * r.normal();
    double ptErr = p.pt * relPt;
    double etaErr = 0.002;
    // State at the last seed hit: radius 16 cm or |z| = 30 cm.
    double t = 0.0;
    double tR;
    bool okR = crossRadius(h, 16.0, tR);
    double tZ = (h.tanL != 0.0) ? ((h.tanL > 0 ? 30.0 : -30.0) - h.vz) / (h.R * h.tanL) : 1e9;
    t = okR ? std::min(tR, tZ) : tZ;
    if (!(t > 0 && t < kPi))
      t = 0.05;
    if (shifted)
      t *= 0.8;  // duplicate seed: last hit one layer earlier
    double pos[3];
    h.at(t, pos);
    double phiT = h.phiAt(t);
    double pxLH = scale * p.pt * std::cos(phiT), pyLH = scale * p.pt * std::sin(phiT), pzLH = spz;

    // TVector3-like helpers (double precision).
    auto ptOf = [](double x, double y) { return std::sqrt(x * x + y * y); };
    auto etaOf = [](double x, double y, double z) {
      double mag = std::sqrt(x * x + y * y + z * z);
      double ct = mag == 0.0 ? 1.0 : z / mag;
      if (ct * ct < 1.0)
        return -0.5 * std::log((1.0 - ct) / (1.0 + ct));
      return z >= 0 ? 10e10 : -10e10;
    };
    auto phiOf = [](double x, double y) { return (x == 0.0 && y == 0.0) ? 0.0 : std::atan2(y, x); };
    auto mpi = [](double a) {
      while (a >= kPi)
        a -= 2 * kPi;
      while (a < -kPi)
        a += 2 * kPi;
      return a;
    };

    {
      const double raw[13] = {spx, spy, spz, dxy, dz, ptErr, etaErr, pos[0], pos[1], pos[2], pxLH, pyLH, pzLH};
      for (int k = 0; k < 13; ++k)
        ev.see_f[k].push_back(f32(raw[k]));
      ev.see_q.push_back(static_cast<int>(p.q));
      ev.see_sim.push_back(particle);
      for (int k = 0; k < (nHits > 3 ? 4 : 3); ++k)
        ev.see_hitIdx.push_back(static_cast<int>(pixBase + k));
      ev.see_hitOff.push_back(static_cast<uint32_t>(ev.see_hitIdx.size()));
    }
    float ptIn = f32(ptOf(pxLH, pyLH));
    float eta = f32(etaOf(pxLH, pyLH, pzLH));
    float fPtErr = f32(ptErr);
    if (!(ptIn > 0.8 - 2 * fPtErr))
      return;
    // r3 at the PCA from (p3PCA, dxy, dz), code/core/trkCore.cc:546-555.
    float ptP = f32(ptOf(spx, spy));
    float pP = f32(std::sqrt(spx * spx + spy * spy + spz * spz));
    float fdxy = f32(dxy), fdz = f32(dz);
    float vz = fdz * ptP * ptP / pP / pP;
    float vx = -fdxy * f32(spy) / ptP - f32(spx) / pP * f32(spz) / pP * fdz;
    float vy = fdxy * f32(spx) / ptP - f32(spy) / pP * f32(spz) / pP * fdz;
    float dPhiChange = f32(mpi(phiOf(pos[0], pos[1]) - phiOf(pxLH, pyLH)));
    int pixtype;
    if (ptIn >= 2.0)
      pixtype = 0;
    else if (ptIn >= (0.8 - 2 * fPtErr) and ptIn < 2.0)
      pixtype = dPhiChange >= 0 ? 1 : 2;
    else
      return;

    bool quad = nHits > 3;
    uint32_t base = static_cast<uint32_t>(ev.x.size());
    uint32_t hit0 = base, hit1 = base + 1, hit2 = base + 2, hit3 = quad ? base + 3 : base + 2;
    float p3PCA_Eta = f32(etaOf(spx, spy, spz));
    float p3PCA_Phi = f32(phiOf(spx, spy));
    auto push = [&](float a, float b, float c, uint32_t pix) {
      ev.x.push_back(a);
      ev.y.push_back(b);
      ev.z.push_back(c);
      ev.detId.push_back(1u);
      ev.idx.push_back(pix);
      ev.simIdx.push_back(particle);
    };
    push(vx, vy, vz, pixBase + 0);
    push(ptP, p3PCA_Eta, p3PCA_Phi, pixBase + 1);
    push(f32(pos[0]), f32(pos[1]), f32(pos[2]), pixBase + 2);
    if (quad)
      push(f32(pos[0]), fdxy, fdz, pixBase + 3);

    ev.h0.push_back(hit0);
    ev.h1.push_back(hit1);
    ev.h2.push_back(hit2);
    ev.h3.push_back(hit3);
    ev.dPhiChange.push_back(dPhiChange);
    ev.ptIn.push_back(ptIn);
    ev.ptErr.push_back(fPtErr);
    ev.px.push_back(f32(pxLH));
    ev.py.push_back(f32(pyLH));
    ev.pz.push_back(f32(pzLH));
    ev.eta.push_back(eta);
    ev.etaErr.push_back(f32(etaErr));
    ev.phi.push_back(f32(phiOf(pxLH, pyLH)));
    ev.charge.push_back(static_cast<int>(p.q));
    ev.seedIdx.push_back(static_cast<uint32_t>(ev.seedIdx.size()));
    float neta = 25., nphi = 72., nz = 25.;
    int etabin = (p3PCA_Eta + 2.6) / ((2 * 2.6) / neta);
    int phibin = (p3PCA_Phi + 3.14159265358979323846) / ((2. * 3.14159265358979323846) / nphi);
    int dzbin = (fdz + 30) / (2 * 30 / nz);
    int isuperbin = (nz * nphi) * etabin + (nz)*phibin + dzbin;
    ev.superbin.push_back(isuperbin);
    ev.pixelType.push_back(static_cast<int8_t>(pixtype));
    ev.isQuad.push_back(quad ? 1 : 0);
    ev.plsSim.push_back(particle);
  }

  void quantize(const Sensor& s, Rng& r, double lu, double lv, double& qu, double& qv) {
    // Centre of the crossed strip row / macro-pixel along u; Gaussian smear along v.
    double k = std::floor((lu + s.halfU) / s.rowU);
    qu = -s.halfU + (k + 0.5) * s.rowU;
    qv = lv + s.sigmaV * r.normal();
  }

  Event* generate(const Geometry& g, const Config& cfg, uint64_t seed) {
    Rng r(seed);
    auto* ev = new Event();
    makeParticles(cfg, r, ev->particles);

    std::vector<SimHit> sim;
    sim.reserve(ev->particles.size() * 16);
    for (int i = 0; i < (int)ev->particles.size(); ++i) {
      auto& p = ev->particles[i];
      Helix h(p.pt, p.eta, p.phi, p.vx, p.vy, p.vz, p.q);
      propagate(g, h, i, sim);
    }
    // Noise hits: 1% of the signal hits, uniform over sensors.
    size_t nNoise = sim.size() / 100;
    for (size_t k = 0; k < nNoise; ++k) {
      int si = int(r.uniform() * g.sensors.size()) % int(g.sensors.size());
      auto& s = g.sensors[si];
      sim.push_back(SimHit{r.uniform(-s.halfU, s.halfU), r.uniform(-s.halfV, s.halfV), si, -1});
    }
    // Outer-tracker hits grouped by sensor (the reference derives per-module hit
    // ranges from the first and last hit index of each module, SDL/Hit.h:255-262).
    std::stable_sort(sim.begin(), sim.end(), [&](const SimHit& a, const SimHit& b) {
      return g.sensors[a.sensor].detId < g.sensors[b.sensor].detId;
    });
    for (auto& h : sim) {
      auto& s = g.sensors[h.sensor];
      double qu, qv;
      quantize(s, r, h.lu, h.lv, qu, qv);
      double pos[3];
      for (int i = 0; i < 3; ++i)
        pos[i] = s.c[i] + qu * s.u[i] + qv * s.v[i];
      ev->x.push_back(f32(pos[0]));
      ev->y.push_back(f32(pos[1]));
      ev->z.push_back(f32(pos[2]));
      ev->detId.push_back(s.detId);
      ev->idx.push_back(static_cast<uint32_t>(ev->idx.size()));
      ev->simIdx.push_back(h.particle);
    }
    ev->nOT = static_cast<uint32_t>(ev->x.size());

    // Pixel seeds.  Every particle above 0.6 GeV inside the pixel acceptance
    // seeds a pLS from its first 3 or 4 inner-tracker hits.  As pixel seeding
    // does, a particle is often seeded more than once: a triplet ending one
    // layer earlier (half of the particles) and, for quadruplets, the outer
    // triplet (half of them), each sharing three pixel hits with the first
    // seed.  Fake seeds, hits of different particles that happen to line up,
    // come in at half the rate of seeded particles: a seeded particle's
    // direction turned by a few mrad, a pT off by a log-normal factor and a
    // random charge, on pixel hits of their own, with no particle (-1).
    // Seeds below the reference's pLS pT cut are dropped by addSeed.
    uint32_t pixHit = 0;
    std::vector<int> seeded;
    for (int i = 0; i < (int)ev->particles.size(); ++i) {
      auto& p = ev->particles[i];
      if (p.pt < 0.6 || std::fabs(p.eta) > 2.6)
        continue;
      seeded.push_back(i);
      Helix h(p.pt, p.eta, p.phi, p.vx, p.vy, p.vz, p.q);
      int nHits = r.uniform() < 0.75 ? 4 : 3;
      uint32_t base = pixHit;
      pixHit += 4;
      addSeed(*ev, h, p, i, r, base, nHits, false);
      if (r.uniform() < 0.5)  // duplicate: the first three hits, last one a layer earlier
        addSeed(*ev, h, p, i, r, base, 3, true);
      if (nHits == 4 && r.uniform() < 0.5)  // duplicate: the outer three hits of the quadruplet
        addSeed(*ev, h, p, i, r, base + 1, 3, false);
    }
    size_t nFake = seeded.size() / 2;
    for (size_t k = 0; k < nFake; ++k) {
      Particle f = ev->particles[seeded[size_t(r.uniform() * seeded.size()) % seeded.size()]];
      f.phi += 0.005 * r.normal();
      f.eta += 0.005 * r.normal();
      f.pt *= std::exp(0.3 * r.normal());
      f.q = r.uniform() < 0.5 ? -1.0 : 1.0;
      Helix h(f.pt, f.eta, f.phi, f.vx, f.vy, f.vz, f.q);
      uint32_t base = pixHit;
      pixHit += 4;
      addSeed(*ev, h, f, -1, r, base, r.uniform() < 0.5 ? 4 : 3, false);
    }
    return ev;
  }

  struct Generator {
    Geometry geo;
  };

}  // namespace

extern "C" {

void* lstgen_create(const char* geometry_dir) {
  auto* g = new Generator();
  if (!buildGeometry(geometry_dir, g->geo)) {
    delete g;
    return nullptr;
  }
  return g;
}

void lstgen_free(void* gen) { delete static_cast<Generator*>(gen); }

// config: 1 single muon, 2 PU200-shaped, 3 PU U(140,250), 5 PU250 + 5% displaced.
// pileup_override > 0 replaces the configuration's pileup mean.
void* lstgen_event(void* gen, int config, unsigned long long seed, double pileup_override) {
  auto* g = static_cast<Generator*>(gen);
  Config cfg{config, 200.0, false, 0.0};
  if (config == 3)
    cfg.pileupRandom = true;
  if (config == 5) {
    cfg.pileup = 250.0;
    cfg.displacedFrac = 0.05;
  }
  if (pileup_override > 0) {
    cfg.pileup = pileup_override;
    cfg.pileupRandom = false;
  }
  return generate(g->geo, cfg, seed);
}

void lstgen_event_free(void* ev) { delete static_cast<Event*>(ev); }

void lstgen_event_sizes(void* ev, unsigned int* nHits, unsigned int* nOT, unsigned int* nPLS, unsigned int* nParticles) {
  auto* e = static_cast<Event*>(ev);
  *nHits = static_cast<unsigned int>(e->x.size());
  *nOT = e->nOT;
  *nPLS = static_cast<unsigned int>(e->ptIn.size());
  *nParticles = static_cast<unsigned int>(e->particles.size());
}

void lstgen_event_hits(
    void* ev, float* x, float* y, float* z, unsigned int* detId, unsigned int* idx, int* simIdx) {
  auto* e = static_cast<Event*>(ev);
  size_t n = e->x.size();
  std::memcpy(x, e->x.data(), n * 4);
  std::memcpy(y, e->y.data(), n * 4);
  std::memcpy(z, e->z.data(), n * 4);
  std::memcpy(detId, e->detId.data(), n * 4);
  std::memcpy(idx, e->idx.data(), n * 4);
  std::memcpy(simIdx, e->simIdx.data(), n * 4);
}

void lstgen_event_pls(void* ev,
                      unsigned int* h0,
                      unsigned int* h1,
                      unsigned int* h2,
                      unsigned int* h3,
                      float* dPhiChange,
                      float* ptIn,
                      float* ptErr,
                      float* px,
                      float* py,
                      float* pz,
                      float* eta,
                      float* etaErr,
                      float* phi,
                      int* charge,
                      unsigned int* seedIdx,
                      int* superbin,
                      signed char* pixelType,
                      char* isQuad,
                      int* simIdx) {
  auto* e = static_cast<Event*>(ev);
  size_t n = e->ptIn.size();
  std::memcpy(h0, e->h0.data(), n * 4);
  std::memcpy(h1, e->h1.data(), n * 4);
  std::memcpy(h2, e->h2.data(), n * 4);
  std::memcpy(h3, e->h3.data(), n * 4);
  std::memcpy(dPhiChange, e->dPhiChange.data(), n * 4);
  std::memcpy(ptIn, e->ptIn.data(), n * 4);
  std::memcpy(ptErr, e->ptErr.data(), n * 4);
  std::memcpy(px, e->px.data(), n * 4);
  std::memcpy(py, e->py.data(), n * 4);
  std::memcpy(pz, e->pz.data(), n * 4);
  std::memcpy(eta, e->eta.data(), n * 4);
  std::memcpy(etaErr, e->etaErr.data(), n * 4);
  std::memcpy(phi, e->phi.data(), n * 4);
  std::memcpy(charge, e->charge.data(), n * 4);
  std::memcpy(seedIdx, e->seedIdx.data(), n * 4);
  std::memcpy(superbin, e->superbin.data(), n * 4);
  std::memcpy(pixelType, e->pixelType.data(), n);
  std::memcpy(isQuad, e->isQuad.data(), n);
  std::memcpy(simIdx, e->plsSim.data(), n * 4);
}

// CMSSW-layout seeds (all of them, before the pT cut): sizes, then the 13
// float arrays see_px .. see_stateTrajGlbPz (each n_seeds), see_q, the
// see_hitIdx offsets (n_seeds + 1) and values, and the seeds' particle index.
void lstgen_event_seed_sizes(void* ev, unsigned int* nSeeds, unsigned int* nSeedHits) {
  auto* e = static_cast<Event*>(ev);
  *nSeeds = static_cast<unsigned int>(e->see_q.size());
  *nSeedHits = static_cast<unsigned int>(e->see_hitIdx.size());
}

void lstgen_event_seeds(void* ev, float* const* f13, int* q, unsigned int* hitOff, int* hitIdx, int* sim) {
  auto* e = static_cast<Event*>(ev);
  size_t n = e->see_q.size();
  for (int k = 0; k < 13; ++k)
    std::memcpy(f13[k], e->see_f[k].data(), n * 4);
  std::memcpy(q, e->see_q.data(), n * 4);
  std::memcpy(hitOff, e->see_hitOff.data(), (n + 1) * 4);
  std::memcpy(hitIdx, e->see_hitIdx.data(), e->see_hitIdx.size() * 4);
  std::memcpy(sim, e->see_sim.data(), n * 4);
}

void lstgen_event_particles(void* ev, double* out7) {
  auto* e = static_cast<Event*>(ev);
  for (size_t i = 0; i < e->particles.size(); ++i) {
    auto& p = e->particles[i];
    double v[7] = {p.pt, p.eta, p.phi, p.q, p.vx, p.vy, p.vz};
    std::memcpy(out7 + 7 * i, v, sizeof(v));
  }
}

}  // extern "C"
