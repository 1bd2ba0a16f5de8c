// Seed conversion of LST::prepareInput (SDL/LST.cc:175-365) on the device:
// CMSSW pixel seeds and outer-tracker hits in, the inputs of
// addHitToEvent + addPixelSegmentToEvent out, written straight into an event
// slot.
//
// Per seed the reference builds three ROOT XYZVectors (double components from
// the float inputs): p3LH (momentum at the last hit), r3LH (its position) and
// p3PCA (momentum at the point of closest approach).  A seed is kept when
// |p3LH|_T > 0.8 - 2 ptErr; it then contributes a pixel line segment and three
// (triplet) or four (quadruplet) pseudo-hits appended after the outer-tracker
// hits, in seed order:
//   hit 0  r3PCA from (p3PCA, dxy, dz)             (calculateR3FromPCA, :163-173)
//   hit 1  (pT, eta, phi) of p3PCA
//   hit 2  r3LH
//   hit 3  (r3LH.x, dxy, dz), quadruplets only; triplets repeat hit 2 as their
//          fourth pLS hit
// with detId 1 and the seed's pixel-hit indices as their ntuple indices.  The
// pLS carries pT, eta, phi, px, py, pz of p3LH, the seed's errors and charge,
// its seed index, the (eta, phi, dz) superbin of p3PCA and a pixel type from
// pT and the sign of "deltaPhi" = phi(r3LH - p3LH) (LST.cc:265, kept as the
// reference computes it; the standalone driver code/core/trkCore.cc:697 uses
// phi(r3LH) - phi(p3LH) instead).
//
// The XYZVector quantities follow ROOT GenVector (Cartesian3D<double>): rho =
// sqrt(x^2 + y^2), r = sqrt(x^2 + y^2 + z^2), phi = atan2(y, x) (0 at the
// origin), eta = asinh(z/rho) as log(z/rho + sqrt((z/rho)^2 + 1)) below
// |z/rho| = 2^13 and its first-order expansion above, +-(|z| + etaMax) on the
// beam line.  All of it is computed in double with separate multiplies and
// adds (the library is built without FMA contraction) and rounded to float
// where the reference stores a float; sqrt and division are IEEE in both, so
// only log and atan2 can differ from the host's libm in the last double bit,
// which survives the rounding to float only within 2^-29 of a float midpoint.
//
// Layout: one block per event converts the seeds in chunks of blockDim.x
// (a block scan of kept-seed and pseudo-hit counts gives the output slots in
// seed order); the other blocks of the event copy the outer-tracker hits.
#pragma once

#include "lst_device.h"

namespace lst {

  constexpr unsigned int kSeedMagic = 0x4453534cu;  // header word 3 of a packed seed event
  constexpr int kSeedFloatArrays = 13;
  // Float seed arrays in LST::run's argument order (SDL/LST.h:35-47).
  enum SeedFloat {
    kSeePx,
    kSeePy,
    kSeePz,
    kSeeDxy,
    kSeeDz,
    kSeePtErr,
    kSeeEtaErr,
    kSeeX,
    kSeeY,
    kSeeZ,
    kSeeTrajPx,
    kSeeTrajPy,
    kSeeTrajPz,
  };

  // Byte layout of one packed seed event (lst_seed_packed_size): a 16-byte
  // header {nPh2, nSeeds, nSeedHits, kSeedMagic}, the outer-tracker hits
  // (detId, x, y, z), the 13 float seed arrays, see_q, the see_hitIdx offsets
  // (nSeeds + 1) and values.  Every array is 4-byte aligned.
  struct SeedLayout {
    size_t detId, x, y, z, f[kSeedFloatArrays], q, hitOff, hitIdx, end;
  };
  LST_HD SeedLayout seedLayout(unsigned int nPh2, unsigned int nSeeds, unsigned int nSeedHits) {
    SeedLayout L;
    size_t o = 16;
    const size_t h4 = 4 * size_t(nPh2), s4 = 4 * size_t(nSeeds);
    L.detId = o; o += h4;
    L.x = o; o += h4;
    L.y = o; o += h4;
    L.z = o; o += h4;
    for (int k = 0; k < kSeedFloatArrays; ++k) {
      L.f[k] = o;
      o += s4;
    }
    L.q = o; o += s4;
    L.hitOff = o; o += s4 + 4;
    L.hitIdx = o; o += 4 * size_t(nSeedHits);
    L.end = (o + 15) & ~size_t(15);
    return L;
  }

#ifdef __CUDACC__
  // ---------------------------------------------------- GenVector in double
  struct Vec3d {
    double x, y, z;
  };
  // log(LDBL_MAX / 256) - log(LDBL_TRUE_MIN * 256) + 16 log 2 for the x87
  // 80-bit long double of the hosts the reference runs on, rounded to double.
  constexpr double kGenVectorEtaMax = 22755.328790602445;

  __device__ __forceinline__ double gvRho(const Vec3d& v) { return sqrt(v.x * v.x + v.y * v.y); }
  __device__ __forceinline__ double gvR(const Vec3d& v) { return sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
  __device__ __forceinline__ double gvPhi(const Vec3d& v) {
    return (v.x == 0.0 && v.y == 0.0) ? 0.0 : atan2(v.y, v.x);
  }
  __device__ __forceinline__ double gvEta(const Vec3d& v) {
    const double rho = gvRho(v);
    if (rho > 0) {
      const double zs = v.z / rho;
      if (fabs(zs) < 8192.0)  // epsilon(double)^(-1/4)
        return log(zs + sqrt(zs * zs + 1.0));
      return v.z > 0 ? log(2.0 * zs + 0.5 / zs) : -log(-2.0 * zs);
    }
    if (v.z == 0)
      return 0;
    return v.z > 0 ? v.z + kGenVectorEtaMax : v.z - kGenVectorEtaMax;
  }

  // Seed conversion of slots blockIdx.y from the packed seed events in blobs.
  // Block 0 of each event converts the seeds; blocks 1.. copy the hits.
  // The host has checked that every blob's 16-byte header lies inside the
  // totalBytes uploaded; a blob whose arrays would end beyond it, or without
  // the seed-event tag, leaves its slot empty with LST_STATUS_INVALID_INPUT.
  __global__ void __launch_bounds__(1024) kPrepareInput(const EventView* evs, const unsigned char* blobs,
                                                        const unsigned long long* offsets,
                                                        unsigned long long totalBytes) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned char* b = blobs + offsets[blockIdx.y];
    const unsigned int* hdr = reinterpret_cast<const unsigned int*>(b);
    const unsigned int nPh2 = hdr[0], nSeeds = hdr[1], nSeedHits = hdr[2];
    const bool badHeader = hdr[3] != kSeedMagic ||
                           offsets[blockIdx.y] + seedLayout(nPh2, nSeeds, nSeedHits).end > totalBytes;
    const bool tooMany = nPh2 > ev.maxHits;
    const SeedLayout L = seedLayout(badHeader ? 0u : nPh2, badHeader ? 0u : nSeeds, badHeader ? 0u : nSeedHits);

    if (blockIdx.x > 0) {
      if (badHeader || tooMany)
        return;
      const float* x = reinterpret_cast<const float*>(b + L.x);
      const float* y = reinterpret_cast<const float*>(b + L.y);
      const float* z = reinterpret_cast<const float*>(b + L.z);
      const unsigned int* det = reinterpret_cast<const unsigned int*>(b + L.detId);
      const unsigned int stride = (gridDim.x - 1) * blockDim.x;
      for (unsigned int i = (blockIdx.x - 1) * blockDim.x + threadIdx.x; i < nPh2; i += stride) {
        ev.hits.xs[i] = x[i];
        ev.hits.ys[i] = y[i];
        ev.hits.zs[i] = z[i];
        ev.hits.detid[i] = det[i];
        ev.hits.idxs[i] = i;
      }
      return;
    }

    __shared__ unsigned int sInvalid;
    if (threadIdx.x == 0)
      sInvalid = 0;
    __syncthreads();
    const unsigned int seeds = (badHeader || tooMany) ? 0u : nSeeds;
    const float* F[kSeedFloatArrays];
#pragma unroll
    for (int k = 0; k < kSeedFloatArrays; ++k)
      F[k] = reinterpret_cast<const float*>(b + L.f[k]);
    const int* q = reinterpret_cast<const int*>(b + L.q);
    const unsigned int* hitOff = reinterpret_cast<const unsigned int*>(b + L.hitOff);
    const int* hitIdx = reinterpret_cast<const int*>(b + L.hitIdx);

    unsigned int runPLS = 0, runPseudo = 0;
    for (unsigned int base = 0; base < seeds; base += blockDim.x) {
      const unsigned int i = base + threadIdx.x;
      bool keep = false;
      unsigned int nPseudo = 0, h0 = 0;
      float ptIn = 0.f, ptErr = 0.f;
      Vec3d p3LH{0, 0, 0};
      if (i < seeds) {
        p3LH = Vec3d{F[kSeeTrajPx][i], F[kSeeTrajPy][i], F[kSeeTrajPz][i]};
        ptIn = static_cast<float>(gvRho(p3LH));
        ptErr = F[kSeePtErr][i];
        keep = static_cast<double>(ptIn) > 0.8 - static_cast<double>(2 * ptErr);
        if (keep) {
          h0 = hitOff[i];
          const unsigned int h1 = hitOff[i + 1];
          if (h1 < h0 || h1 > nSeedHits || h1 - h0 < 3) {
            keep = false;  // the reference reads three pixel hits of every kept seed
            atomicOr(&sInvalid, 1u);
          } else {
            nPseudo = h1 - h0 > 3 ? 4u : 3u;
          }
        }
      }
      // Kept seeds below 2^16 per chunk, pseudo-hits in the upper half.
      unsigned int chunkTotal;
      const unsigned int ex = blockExclusiveScan((nPseudo << 16) | (keep ? 1u : 0u), chunkTotal);
      if (keep) {
        const unsigned int pls = runPLS + (ex & 0xffffu);
        const unsigned int hit = nPh2 + runPseudo + (ex >> 16);
        const bool quad = nPseudo == 4;
        const float dxy = F[kSeeDxy][i], dz = F[kSeeDz][i];
        const Vec3d r3LH{F[kSeeX][i], F[kSeeY][i], F[kSeeZ][i]};
        const Vec3d p3PCA{F[kSeePx][i], F[kSeePy][i], F[kSeePz][i]};
        // calculateR3FromPCA
        const float pt = static_cast<float>(gvRho(p3PCA));
        const float p = static_cast<float>(gvR(p3PCA));
        const float vz = dz * pt * pt / p / p;
        const float vx = static_cast<float>(static_cast<double>(-dxy) * p3PCA.y / static_cast<double>(pt) -
                                            p3PCA.x / static_cast<double>(p) * p3PCA.z / static_cast<double>(p) *
                                                static_cast<double>(dz));
        const float vy = static_cast<float>(static_cast<double>(dxy) * p3PCA.x / static_cast<double>(pt) -
                                            p3PCA.y / static_cast<double>(p) * p3PCA.z / static_cast<double>(p) *
                                                static_cast<double>(dz));
        const float dPhiChange = static_cast<float>(gvPhi(Vec3d{r3LH.x - p3LH.x, r3LH.y - p3LH.y, r3LH.z - p3LH.z}));
        const float pcaPt = static_cast<float>(gvRho(p3PCA));
        const float pcaEta = static_cast<float>(gvEta(p3PCA));
        const float pcaPhi = static_cast<float>(gvPhi(p3PCA));
        if (hit + nPseudo <= ev.maxHits) {
          const float hx[4] = {vx, pcaPt, F[kSeeX][i], F[kSeeX][i]};
          const float hy[4] = {vy, pcaEta, F[kSeeY][i], dxy};
          const float hz[4] = {vz, pcaPhi, F[kSeeZ][i], dz};
          for (unsigned int k = 0; k < nPseudo; ++k) {
            ev.hits.xs[hit + k] = hx[k];
            ev.hits.ys[hit + k] = hy[k];
            ev.hits.zs[hit + k] = hz[k];
            ev.hits.detid[hit + k] = 1u;
            ev.hits.idxs[hit + k] = static_cast<unsigned int>(hitIdx[h0 + k]);
          }
        }
        if (pls < kMaxPixelSegments) {
          const float neta = 25.f, nphi = 72.f, nz = 25.f;
          const int etabin = static_cast<int>((static_cast<double>(pcaEta) + 2.6) / ((2 * 2.6) / neta));
          const int phibin = static_cast<int>((static_cast<double>(pcaPhi) + 3.14159265358979323846) /
                                              ((2. * 3.14159265358979323846) / nphi));
          const int dzbin = static_cast<int>((dz + 30) / (2 * 30 / nz));
          const int superbin = static_cast<int>((nz * nphi) * etabin + (nz)*phibin + dzbin);
          ev.plsHit0[pls] = hit;
          ev.plsHit1[pls] = hit + 1;
          ev.plsHit2[pls] = hit + 2;
          ev.plsHit3[pls] = quad ? hit + 3 : hit + 2;
          ev.plsDPhiChange[pls] = dPhiChange;
          ev.ls.ptIn[pls] = ptIn;
          ev.ls.ptErr[pls] = ptErr;
          ev.ls.px[pls] = F[kSeeTrajPx][i];
          ev.ls.py[pls] = F[kSeeTrajPy][i];
          ev.ls.pz[pls] = F[kSeeTrajPz][i];
          ev.ls.eta[pls] = static_cast<float>(gvEta(p3LH));
          ev.ls.etaErr[pls] = F[kSeeEtaErr][i];
          ev.ls.phi[pls] = static_cast<float>(gvPhi(p3LH));
          ev.ls.charge[pls] = q[i];
          ev.ls.seedIdx[pls] = i;
          ev.ls.superbin[pls] = superbin;
          ev.ls.pixelType[pls] = static_cast<int8_t>(ptIn >= 2.0 ? 0 : (dPhiChange >= 0 ? 1 : 2));
          ev.ls.isQuad[pls] = quad ? 1 : 0;
        }
      }
      runPLS += chunkTotal & 0xffffu;
      runPseudo += chunkTotal >> 16;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned int status = 0;
      unsigned int nHits = nPh2 + runPseudo, nPLS = runPLS;
      if (badHeader || sInvalid)
        status |= kStatusInvalidInput;
      if (badHeader) {
        nHits = 0;
        nPLS = 0;
      } else if (tooMany || nHits > ev.maxHits) {
        status |= kStatusHitCapacity;
        nHits = 0;
        nPLS = 0;
      }
      if (nPLS > kMaxPixelSegments) {
        status |= kStatusPLSTruncated;
        nPLS = kMaxPixelSegments;
      }
      ev.sc->nHits = nHits;
      ev.sc->nPLS = nPLS;
      ev.sc->status |= status;
    }
  }
#endif

}  // namespace lst
