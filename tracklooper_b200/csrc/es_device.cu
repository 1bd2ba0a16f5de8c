// Event-setup build on the device.  The host reads the geometry files as raw
// records and computes one value per sensor, its eta (the reference's host
// build takes acosh in float through the C library, SDL/ModuleMethods.h:218,
// and the device build keeps that value); everything else of the event setup
// is built by the kernels below and then copied back into the host mirror:
//
//  * module re-indexing in ascending detId order, lower modules first, the
//    pixel module next, upper modules last (SDL/ModuleMethods.h:285-366), with
//    the detId fields, types and r of each module;
//  * the detId -> module hash (the host loader's open-addressing table,
//    inserted in the same order, so the table is identical);
//  * endcap and tilted-barrel orientations, a later record of a detId
//    replacing an earlier one (SDL/EndcapGeometry.cc:13-41,
//    SDL/TiltedGeometry.cc:5-33), and the sorted endcap orientation map;
//  * partner modules and the drdz / dxdy taken from the partner
//    (SDL/ModuleMethods.h:368-382), in ascending detId order;
//  * the module connection map and the pixel-seed module maps, framed from
//    the raw {key, n, n x detId} records as SDL/ModuleConnectionMap.cc:9-50
//    reads them (SDL/ModuleMethods.h:33-141);
//  * the static occupancy caps and arena offsets (SDL/MiniDoublet.h:994-1082,
//    SDL/Segment.h:912-1008, SDL/Triplet.h:1007-1102,
//    SDL/Quintuplet.h:3117-3213).
//
// Errors are reported with the messages of the host loader (csrc/es.cc) and
// in its order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "es.h"
#include "lst_core.h"
#include "lst_md.h"

namespace lst {

  namespace esb {

    constexpr unsigned int kNone = 0xffffffffu;
    constexpr int kPixFiles = 12;
    constexpr unsigned int kPixKeys = 2 * kSizeSuperbins;  // charge-inclusive keys are offset by 45000

    struct Status {
      unsigned int dup;             // two sensors share a detId
      unsigned int reserved;        // a sensor has detId 1
      unsigned int nLower;          // lower sensors found
      unsigned int partnerMissing;  // detId whose partner is missing (first in detId order)
      unsigned int connBad;         // smallest detId with a bad connection record
      unsigned int pixSizeBad;      // smallest 3 sb + charge with more than 80 modules
      unsigned long long pixUnknown;  // smallest (position << 32 | detId) of an unknown pixel-map entry
      unsigned int geoCount;        // endcap orientation map entries
      unsigned int nRec[1 + kPixFiles];  // records framed per map file
      unsigned int pixTotal[3];
      int mdTotal, lsTotal;
      unsigned int t3Total, t5Total;
    };

    __device__ __forceinline__ unsigned int hashFind(const unsigned int* key, const uint16_t* val, unsigned int bits,
                                                     unsigned int detId) {
      const unsigned int mask = (1u << bits) - 1;
      unsigned int slot = (detId * 2654435761u) >> (32 - bits);
      for (unsigned int probe = 0; probe <= mask; ++probe) {
        const uint16_t v = val[slot];
        if (v == 0xffff)
          return kNone;
        if (key[slot] == detId)
          return v;
        slot = (slot + 1) & mask;
      }
      return kNone;
    }

    // Block-wide exclusive scan of one value per thread (blockDim.x = 1024).
    __device__ unsigned int blockScan(unsigned int v, unsigned int& total) {
      __shared__ unsigned int warpSums[32];
      const unsigned int lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
      unsigned int incl = v;
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (int(lane) >= o)
          incl += y;
      }
      __syncthreads();
      if (lane == 31)
        warpSums[warp] = incl;
      __syncthreads();
      if (warp == 0) {
        unsigned int s = warpSums[lane];
        for (int o = 1; o < 32; o <<= 1) {
          const unsigned int y = __shfl_up_sync(0xffffffffu, s, o);
          if (int(lane) >= o)
            s += y;
        }
        warpSums[lane] = s;
      }
      __syncthreads();
      total = warpSums[31];
      return incl - v + (warp ? warpSums[warp - 1] : 0u);
    }

    // Rank of every key among all keys (they are unique in a valid file), and
    // the keys in ascending order with their source positions.
    __global__ void kRank(const unsigned int* keys, unsigned int n, unsigned int* sorted, unsigned int* srcOf,
                          Status* st) {
      __shared__ unsigned int tile[1024];
      const unsigned int p = blockIdx.x * blockDim.x + threadIdx.x;
      const unsigned int k = p < n ? keys[p] : 0u;
      unsigned int less = 0, equal = 0;
      for (unsigned int t0 = 0; t0 < n; t0 += blockDim.x) {
        __syncthreads();
        if (t0 + threadIdx.x < n)
          tile[threadIdx.x] = keys[t0 + threadIdx.x];
        __syncthreads();
        const unsigned int m = min(blockDim.x, n - t0);
        for (unsigned int j = 0; j < m; ++j) {
          const unsigned int o = tile[j];
          less += o < k;
          equal += o == k;
        }
      }
      if (p < n) {
        if (equal > 1)
          atomicOr(&st->dup, 1u);
        sorted[less] = k;  // with duplicates several keys land on one slot; the build then fails
        srcOf[less] = p;
      }
    }

    __device__ bool isInverted(short subdet, short side, short module, short layer) {
      if (subdet == Endcap) {
        if (side == NegZ)
          return module % 2 == 1;
        if (side == PosZ)
          return module % 2 == 0;
        return false;
      }
      if (subdet == Barrel) {
        if (side == Center) {
          if (layer <= 3)
            return module % 2 == 1;
          if (layer >= 4)
            return module % 2 == 0;
          return false;
        }
        if (side == NegZ or side == PosZ) {
          if (layer <= 2)
            return module % 2 == 1;
          if (layer == 3)
            return module % 2 == 0;
          return false;
        }
        return false;
      }
      return false;
    }

    struct ModuleOut {
      unsigned int* detIds;
      short *layers, *rings, *modules, *rods, *subdets, *sides;
      float *eta, *r;
      uint8_t *isInverted, *isLower, *isAnchor, *moduleType, *moduleLayerType;
      int* sdlLayers;
      unsigned int* mapdetId;
      uint16_t* mapIdx;
    };

    // Module indices and per-module fields; one block walks the sorted detIds.
    __global__ void __launch_bounds__(1024) kModules(const unsigned int* sorted, const unsigned int* srcOf,
                                                     const unsigned int* cent, const float* etaRec, unsigned int nMod,
                                                     unsigned int nLower, ModuleOut o, Status* st) {
      unsigned int lowerCarry = 0, upperCarry = 0;
      for (unsigned int s0 = 0; s0 < nMod; s0 += blockDim.x) {
        const unsigned int s = s0 + threadIdx.x;
        const bool in = s < nMod;
        const unsigned int detId = in ? sorted[s] : 0u;
        const bool pixel = in && detId == 1u;
        short subdet = 0, side = 0, layer = 0, ring = 0, module = 0, rod = 0;
        bool inv = false, low = false;
        if (in && !pixel) {
          subdet = static_cast<short>((detId & (7u << 25)) >> 25);
          side = static_cast<short>(subdet == Endcap ? (detId & (3u << 23)) >> 23 : (detId & (3u << 18)) >> 18);
          layer = static_cast<short>(subdet == Endcap ? (detId & (7u << 18)) >> 18 : (detId & (7u << 20)) >> 20);
          ring = static_cast<short>(subdet == Endcap ? (detId & (15u << 12)) >> 12 : 0);
          module = static_cast<short>((detId & (127u << 2)) >> 2);
          rod = static_cast<short>(subdet == Endcap ? 0 : (detId & (127u << 10)) >> 10);
          inv = isInverted(subdet, side, module, layer);
          low = inv ? !(detId & 1u) : (detId & 1u);
        }
        unsigned int nLowHere, nUpHere;
        const unsigned int lowBefore = blockScan(in && !pixel && low ? 1u : 0u, nLowHere);
        const unsigned int upBefore = blockScan(in && !pixel && !low ? 1u : 0u, nUpHere);
        if (in) {
          unsigned int idx;
          if (pixel)
            idx = nLower;
          else if (low)
            idx = lowerCarry + lowBefore;
          else
            idx = nLower + 1 + upperCarry + upBefore;
          o.mapdetId[s] = detId;
          const bool okIdx = pixel || (low ? idx < nLower : idx < nMod);
          o.mapIdx[s] = okIdx ? static_cast<uint16_t>(idx) : uint16_t(0xffff);
          if (okIdx) {
            o.detIds[idx] = detId;
            if (pixel) {
              o.moduleType[idx] = PixelModule;
              o.moduleLayerType[idx] = InnerPixelLayer;
            } else {
              const unsigned int src = srcOf[s];
              // a centroid record: detId, x, y, z, type
              const float x = __uint_as_float(cent[5 * src + 1]), y = __uint_as_float(cent[5 * src + 2]),
                          z = __uint_as_float(cent[5 * src + 3]);
              const int type = static_cast<int>(cent[5 * src + 4]);
              o.layers[idx] = layer;
              o.rings[idx] = ring;
              o.rods[idx] = rod;
              o.modules[idx] = module;
              o.subdets[idx] = subdet;
              o.sides[idx] = side;
              o.eta[idx] = etaRec[src];
              o.r[idx] = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z)));
              o.isInverted[idx] = inv;
              o.isLower[idx] = low;
              const uint8_t mtype = (type == 25) ? TwoS : PS;
              const uint8_t mltype = (type == 23) ? Pixel : Strip;
              o.moduleType[idx] = mtype;
              o.moduleLayerType[idx] = mltype;
              o.isAnchor[idx] = (mtype == PS && mltype == Pixel) || (mtype == TwoS && low);
              o.sdlLayers[idx] = layer + 6 * (subdet == Endcap) + 5 * (subdet == Endcap && mtype == TwoS);
            }
          }
        }
        lowerCarry += nLowHere;
        upperCarry += nUpHere;
      }
      if (threadIdx.x == 0)
        st->nLower = lowerCarry;
    }

    // The detId hash, filled in ascending detId order as the host loader
    // fills it (one thread: the table's layout depends on the order).
    __global__ void kHash(const unsigned int* mapdetId, const uint16_t* mapIdx, unsigned int nMod, unsigned int bits,
                          unsigned int* hashKey, uint16_t* hashVal) {
      if (blockIdx.x != 0 || threadIdx.x != 0)
        return;
      const unsigned int mask = (1u << bits) - 1;
      for (unsigned int i = 0; i < nMod; ++i) {
        const unsigned int key = mapdetId[i];
        unsigned int slot = (key * 2654435761u) >> (32 - bits);
        for (unsigned int probe = 0; probe <= mask; ++probe) {
          if (hashVal[slot] == 0xffff || hashKey[slot] == key)
            break;
          slot = (slot + 1) & mask;
        }
        hashKey[slot] = key;
        hashVal[slot] = mapIdx[i];
      }
    }

    // Marks the records (stride words each, detId first) that no later record
    // of the same detId replaces.
    __global__ void kLastOfKey(const unsigned int* rec, unsigned int n, unsigned int stride, uint8_t* last) {
      __shared__ unsigned int tile[1024];
      const unsigned int k = blockIdx.x * blockDim.x + threadIdx.x;
      const unsigned int key = k < n ? rec[size_t(k) * stride] : 0u;
      bool replaced = false;
      for (unsigned int t0 = 0; t0 < n; t0 += blockDim.x) {
        __syncthreads();
        if (t0 + threadIdx.x < n)
          tile[threadIdx.x] = rec[size_t(t0 + threadIdx.x) * stride];
        __syncthreads();
        const unsigned int m = min(blockDim.x, n - t0);
        for (unsigned int j = 0; j < m; ++j)
          replaced |= (t0 + j > k) && tile[j] == key;
      }
      if (k < n)
        last[k] = !replaced;
    }

    // The endcap orientation map: the surviving records in detId order, and
    // per module its position in the map.  Also records which record gives
    // each module its orientation.
    __global__ void kOrientIndex(const unsigned int* rec, unsigned int n, const uint8_t* last, bool endcap,
                                 const unsigned int* hashKey, const uint16_t* hashVal, unsigned int bits,
                                 unsigned int* recOfModule, unsigned int* geoDetId, float* geoPhi, int* geoIndex,
                                 Status* st) {
      __shared__ unsigned int tile[1024];
      __shared__ uint8_t tileLast[1024];
      const unsigned int k = blockIdx.x * blockDim.x + threadIdx.x;
      const unsigned int key = k < n ? rec[3 * k] : 0u;
      unsigned int rank = 0;
      if (endcap) {
        for (unsigned int t0 = 0; t0 < n; t0 += blockDim.x) {
          __syncthreads();
          if (t0 + threadIdx.x < n) {
            tile[threadIdx.x] = rec[3 * (t0 + threadIdx.x)];
            tileLast[threadIdx.x] = last[t0 + threadIdx.x];
          }
          __syncthreads();
          const unsigned int m = min(blockDim.x, n - t0);
          for (unsigned int j = 0; j < m; ++j)
            rank += tileLast[j] && tile[j] < key;
        }
      }
      if (k >= n || !last[k])
        return;
      const unsigned int mi = hashFind(hashKey, hashVal, bits, key);
      if (mi != kNone)
        recOfModule[mi] = k;
      if (endcap) {
        geoDetId[rank] = key;
        geoPhi[rank] = __uint_as_float(rec[3 * k + 2]);
        if (mi != kNone)
          geoIndex[mi] = static_cast<int>(rank);
        atomicAdd(&st->geoCount, 1u);
      }
    }

    // dxdy and drdz of each module from its orientation records
    // (SDL/ModuleMethods.h:245-260).
    __global__ void kOrientApply(const unsigned int* endc, const unsigned int* tilt, const unsigned int* endRecOf,
                                 const unsigned int* tiltRecOf, const unsigned int* detIds, const short* subdets,
                                 unsigned int nMod, float* dxdys, float* drdzs) {
      const unsigned int i = blockIdx.x * blockDim.x + threadIdx.x;
      if (i >= nMod || detIds[i] == 1u)
        return;
      if (subdets[i] == Endcap) {
        const unsigned int k = endRecOf[i];
        dxdys[i] = k == kNone ? 0.f : __uint_as_float(endc[3 * k + 1]);
        drdzs[i] = 0.f;
      } else {
        const unsigned int k = tiltRecOf[i];
        dxdys[i] = k == kNone ? 0.f : __uint_as_float(tilt[3 * k + 2]);
        drdzs[i] = (subdets[i] == Barrel && k != kNone) ? __uint_as_float(tilt[3 * k + 1]) : 0.f;
      }
    }

    // Partner modules, and drdz / dxdy taken from the partner where missing,
    // in ascending detId order (one thread: a module may read a partner's
    // value set earlier in the walk, as in the host loader).
    __global__ void kPartners(const unsigned int* mapdetId, const uint16_t* mapIdx, unsigned int nMod,
                              const unsigned int* hashKey, const uint16_t* hashVal, unsigned int bits,
                              const uint8_t* isLower, const uint8_t* isInverted, uint16_t* partner, float* drdzs,
                              float* dxdys, Status* st) {
      if (blockIdx.x != 0 || threadIdx.x != 0)
        return;
      for (unsigned int s = 0; s < nMod; ++s) {
        const unsigned int detId = mapdetId[s];
        if (detId == 1u)
          continue;
        const unsigned int idx = mapIdx[s];
        const bool low = isLower[idx], inv = isInverted[idx];
        const unsigned int pd = low ? (inv ? detId - 1 : detId + 1) : (inv ? detId + 1 : detId - 1);
        const unsigned int p = hashFind(hashKey, hashVal, bits, pd);
        if (p == kNone) {
          st->partnerMissing = detId;
          return;
        }
        partner[idx] = static_cast<uint16_t>(p);
        if (drdzs[idx] == 0)
          drdzs[idx] = drdzs[p];
        if (dxdys[idx] == 0)
          dxdys[idx] = dxdys[p];
      }
    }

    // Frames {key, n, n x u32} records as the host reader does: a record
    // whose count runs past the end of the file ends the file.  One thread
    // per file.
    struct MapFiles {
      const unsigned int* words;
      unsigned long long wordOff[1 + kPixFiles + 1];
      unsigned long long bytes[1 + kPixFiles];
      unsigned int* recKey;
      unsigned int* recN;
      unsigned long long* recStart;
      unsigned long long recOff[1 + kPixFiles + 1];  // record capacity of each file (its words / 2)
    };
    __global__ void kFrame(MapFiles f, Status* st) {
      const unsigned int file = blockIdx.x * blockDim.x + threadIdx.x;
      if (file >= 1 + kPixFiles)
        return;
      const unsigned int* w = f.words + f.wordOff[file];
      const unsigned long long bytes = f.bytes[file];
      unsigned long long pos = 0;  // in words
      unsigned int n = 0;
      const unsigned long long cap = f.recOff[file + 1] - f.recOff[file];
      while ((pos + 2) * 4 <= bytes && n < cap) {
        const unsigned int key = w[pos], cnt = w[pos + 1];
        const unsigned long long left = bytes - (pos + 2) * 4;
        if (static_cast<unsigned long long>(cnt) > left / 4)
          break;
        f.recKey[f.recOff[file] + n] = key;
        f.recN[f.recOff[file] + n] = cnt;
        f.recStart[f.recOff[file] + n] = f.wordOff[file] + pos + 2;
        ++n;
        pos += 2 + static_cast<unsigned long long>(cnt);
      }
      st->nRec[file] = n;
    }

    // The last record of each module's detId in the connection map.
    __global__ void kConnWin(MapFiles f, const Status* st, const unsigned int* hashKey, const uint16_t* hashVal,
                             unsigned int bits, unsigned int* winOfModule) {
      const unsigned int k = blockIdx.x * blockDim.x + threadIdx.x;
      if (k >= st->nRec[0])
        return;
      const unsigned int mi = hashFind(hashKey, hashVal, bits, f.recKey[k]);
      if (mi != kNone)
        atomicMax(&winOfModule[mi], k + 1);
    }

    // A module whose record is bad gets, in errDetail, kNone for too many
    // connections or else the first unknown detId it lists.
    __global__ void kConnApply(MapFiles f, const unsigned int* winOfModule, const unsigned int* detIds,
                               unsigned int nMod, const unsigned int* hashKey, const uint16_t* hashVal,
                               unsigned int bits, uint16_t* nConnected, uint16_t* moduleMap, unsigned int* errDetail,
                               Status* st) {
      const unsigned int i = blockIdx.x * blockDim.x + threadIdx.x;
      if (i >= nMod || winOfModule[i] == 0)
        return;
      const unsigned int k = winOfModule[i] - 1;
      const unsigned int n = f.recN[k];
      if (n > kMaxConnectedModules) {
        errDetail[i] = kNone;
        atomicMin(&st->connBad, detIds[i]);
        return;
      }
      nConnected[i] = static_cast<uint16_t>(n);
      for (unsigned int j = 0; j < n; ++j) {
        const unsigned int d = f.words[f.recStart[k] + j];
        const unsigned int mi = hashFind(hashKey, hashVal, bits, d);
        if (mi == kNone) {
          errDetail[i] = d;
          atomicMin(&st->connBad, detIds[i]);
          return;
        }
        moduleMap[size_t(i) * kMaxConnectedModules + j] = static_cast<uint16_t>(mi);
      }
    }

    // The last record of each key in each pixel map file.
    __global__ void kPixWin(MapFiles f, const Status* st, unsigned int* keyRec) {
      const unsigned int file = blockIdx.y;
      const unsigned int k = blockIdx.x * blockDim.x + threadIdx.x;
      if (k >= st->nRec[1 + file])
        return;
      const unsigned long long r = f.recOff[1 + file] + k;
      const unsigned int key = f.recKey[r];
      if (key < kPixKeys)
        atomicMax(&keyRec[size_t(file) * kPixKeys + key], k + 1);
    }

    __device__ __forceinline__ unsigned int pixKey(int c, unsigned int sb) { return c == 0 ? sb + kSizeSuperbins : sb; }

    // Modules listed for each superbin and charge class.
    __global__ void kPixSizes(MapFiles f, const unsigned int* keyRec, unsigned int* sizes, Status* st) {
      const unsigned int sb = blockIdx.x * blockDim.x + threadIdx.x;
      const int c = blockIdx.y;
      if (sb >= kSizeSuperbins)
        return;
      unsigned int total = 0;
      for (int l = 0; l < 4; ++l) {
        const int file = c * 4 + l;
        const unsigned int w = keyRec[size_t(file) * kPixKeys + pixKey(c, sb)];
        if (w)
          total += f.recN[f.recOff[1 + file] + w - 1];
      }
      sizes[c * kSizeSuperbins + sb] = total;
      if (total > kMaxConnectedModules)
        atomicMin(&st->pixSizeBad, 3 * sb + unsigned(c));
    }

    // Exclusive scan of the superbin sizes per charge class; one block each.
    __global__ void __launch_bounds__(1024) kPixScan(const unsigned int* sizes, unsigned int* index, Status* st) {
      const int c = blockIdx.x;
      unsigned int carry = 0;
      for (unsigned int s0 = 0; s0 < kSizeSuperbins; s0 += blockDim.x) {
        const unsigned int sb = s0 + threadIdx.x;
        const unsigned int v = sb < kSizeSuperbins ? sizes[c * kSizeSuperbins + sb] : 0u;
        unsigned int tot;
        const unsigned int ex = blockScan(v, tot);
        if (sb < kSizeSuperbins)
          index[c * kSizeSuperbins + sb] = carry + ex;
        carry += tot;
      }
      if (threadIdx.x == 0)
        st->pixTotal[c] = carry;
    }

    // connectedPixels: per charge class, per superbin, the four layers' lists.
    __global__ void kPixFill(MapFiles f, const unsigned int* keyRec, const unsigned int* index,
                             const unsigned int* hashKey, const uint16_t* hashVal, unsigned int bits,
                             unsigned int* connectedPixels, unsigned long long capacity, Status* st) {
      const unsigned int sb = blockIdx.x * blockDim.x + threadIdx.x;
      const int c = blockIdx.y;
      if (sb >= kSizeSuperbins)
        return;
      unsigned long long pos = index[c * kSizeSuperbins + sb];
      for (int cc = 0; cc < c; ++cc)
        pos += st->pixTotal[cc];
      for (int l = 0; l < 4; ++l) {
        const int file = c * 4 + l;
        const unsigned int w = keyRec[size_t(file) * kPixKeys + pixKey(c, sb)];
        if (!w)
          continue;
        const unsigned long long r = f.recOff[1 + file] + w - 1;
        const unsigned int n = f.recN[r];
        for (unsigned int j = 0; j < n && pos < capacity; ++j, ++pos) {
          const unsigned int d = f.words[f.recStart[r] + j];
          const unsigned int mi = hashFind(hashKey, hashVal, bits, d);
          if (mi == kNone)
            atomicMin(&st->pixUnknown, (pos << 32) | d);
          else
            connectedPixels[pos] = mi;
        }
      }
    }

    // Static caps and arena offsets; one block walks the lower modules.
    __global__ void __launch_bounds__(1024) kCaps(const short* layers, const short* subdets, const short* rings,
                                                  const float* eta, const uint16_t* nConnected, unsigned int nLower,
                                                  int* mdOffset, int* mdCap, int* lsOffset, int* lsCap, int* t3Cap,
                                                  int* t5Cap, Status* st) {
      __shared__ unsigned int sT3, sT5;
      if (threadIdx.x == 0)
        sT3 = sT5 = 0;
      unsigned int mdCarry = 0, lsCarry = 0;
      for (unsigned int s0 = 0; s0 < nLower; s0 += blockDim.x) {
        const unsigned int i = s0 + threadIdx.x;
        int mdc = 0, lsc = 0;
        if (i < nLower) {
          const int cat = occupancyCategory(layers[i], subdets[i], rings[i]);
          const int etaBin = occupancyEtaBin(fabsf(eta[i]));
          mdc = mdOccupancy(cat, etaBin);
          lsc = nConnected[i] == 0 ? 0 : lsOccupancy(cat, etaBin);
        }
        unsigned int mdTot, lsTot;
        const unsigned int mdEx = blockScan(static_cast<unsigned int>(mdc), mdTot);
        const unsigned int lsEx = blockScan(static_cast<unsigned int>(lsc), lsTot);
        if (i < nLower) {
          const int cat = occupancyCategory(layers[i], subdets[i], rings[i]);
          const int etaBin = occupancyEtaBin(fabsf(eta[i]));
          mdOffset[i] = static_cast<int>(mdCarry + mdEx);
          mdCap[i] = mdc;
          lsOffset[i] = static_cast<int>(lsCarry + lsEx);
          lsCap[i] = lsc;
          const int t3c = t3Occupancy(cat, etaBin);
          t3Cap[i] = t3c;
          if (nConnected[i] != 0)
            atomicAdd(&sT3, static_cast<unsigned int>(t3c));
          const bool eligible =
              !(subdets[i] == Barrel && layers[i] >= 3) && !(subdets[i] == Endcap && layers[i] > 1);
          if (eligible) {
            const int t5c = t5Occupancy(cat, etaBin);
            t5Cap[i] = t5c;
            atomicAdd(&sT5, static_cast<unsigned int>(t5c));
          } else {
            t5Cap[i] = -1;
          }
        }
        mdCarry += mdTot;
        lsCarry += lsTot;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        mdOffset[nLower] = static_cast<int>(mdCarry);
        mdCap[nLower] = static_cast<int>(kMaxPixelMDs);
        lsOffset[nLower] = static_cast<int>(lsCarry);
        lsCap[nLower] = 0;
        st->mdTotal = static_cast<int>(mdCarry);
        st->lsTotal = static_cast<int>(lsCarry);
        st->t3Total = sT3;
        st->t5Total = sT5;
      }
    }

    // ------------------------------------------------------------ host side
    bool readBytes(const std::string& path, std::vector<char>& out) {
      std::ifstream f(path, std::ios::binary | std::ios::ate);
      if (!f.is_open())
        return false;
      const std::streamsize n = f.tellg();
      f.seekg(0);
      out.resize(static_cast<size_t>(n));
      return n == 0 || static_cast<bool>(f.read(out.data(), n));
    }

    // Device allocations of one build, freed together.
    struct Pool {
      std::vector<void*> ptrs;
      ~Pool() {
        for (void* p : ptrs)
          cudaFree(p);
      }
      template <typename T>
      T* get(size_t n, cudaError_t& err) {
        void* p = nullptr;
        if (err == cudaSuccess)
          err = cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T));
        if (err == cudaSuccess)
          ptrs.push_back(p);
        return static_cast<T*>(p);
      }
    };

    template <typename T>
    cudaError_t down(std::vector<T>& v, const T* d, size_t n) {
      v.resize(n);
      return n ? cudaMemcpy(v.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost) : cudaSuccess;
    }

  }  // namespace esb

  std::string buildEsOnDevice(const std::string& dir, int device, EsHost& es) {
    using namespace esb;
    es = EsHost();
    es.ptCut = geometryPtCut(dir);
    // the files, as raw records (the host loader's read order and messages)
    std::vector<char> centB, endB, tiltB, connB;
    if (!readBytes(dir + "/sensor_centroids.bin", centB) || centB.size() < 20)
      return "unable to read " + dir + "/sensor_centroids.bin";
    if (!readBytes(dir + "/endcap_orientation.bin", endB))
      return "unable to read " + dir + "/endcap_orientation.bin";
    if (!readBytes(dir + "/tilted_barrel_orientation.bin", tiltB))
      return "unable to read " + dir + "/tilted_barrel_orientation.bin";
    if (!readBytes(dir + "/module_connection_tracing_merged.bin", connB))
      return "unable to read " + dir + "/module_connection_tracing_merged.bin";
    static const char* kLayers[4] = {"_layer1_subdet5", "_layer2_subdet5", "_layer1_subdet4", "_layer2_subdet4"};
    std::vector<char> pixB[kPixFiles];
    std::string pixMissing;  // reported where the host loader reads these files
    for (int f = 0; f < kPixFiles && pixMissing.empty(); ++f) {
      const int c = f / 4, l = f % 4;
      const char* charge = c == 0 ? "" : (c == 1 ? "_pos" : "_neg");
      const std::string path = dir + "/pixelmap/pLS_map" + charge + kLayers[l] + ".bin";
      if (!readBytes(path, pixB[f]))
        pixMissing = "unable to read " + path;
    }

    // whole records only, as the host reader takes them
    const unsigned int nSens = static_cast<unsigned int>(centB.size() / 20);
    const unsigned int nEnd = static_cast<unsigned int>(endB.size() / 12);
    const unsigned int nTilt = static_cast<unsigned int>(tiltB.size() / 12);
    const unsigned int nMod = nSens + 1;  // + the pixel module (detId 1)
    std::vector<unsigned int> cent(size_t(nSens) * 5);
    std::memcpy(cent.data(), centB.data(), size_t(nSens) * 20);
    // per-sensor eta through the C library's float acosh, as the reference's
    // host build computes it
    std::vector<float> etaRec(nSens);
    std::vector<unsigned int> keys(nMod);
    bool reserved = false;
    for (unsigned int i = 0; i < nSens; ++i) {
      keys[i] = cent[5 * i];
      reserved |= keys[i] == 1u;
      float m_x, m_y, m_z;
      std::memcpy(&m_x, &cent[5 * i + 1], 4);
      std::memcpy(&m_y, &cent[5 * i + 2], 4);
      std::memcpy(&m_z, &cent[5 * i + 3], 4);
      const float r = std::sqrt(m_x * m_x + m_y * m_y + m_z * m_z);
      etaRec[i] = ((m_z > 0) - (m_z < 0)) * std::acosh(r / std::sqrt(m_x * m_x + m_y * m_y));
    }
    keys[nSens] = 1u;
    unsigned int bits = 4;
    while ((1u << bits) < 2u * nMod)
      ++bits;
    const unsigned int nLower = (nMod - 1) / 2;

    // the map files as one word array, each file's words and record slots
    MapFiles mf{};
    const std::vector<char>* files[1 + kPixFiles] = {&connB};
    for (int i = 0; i < kPixFiles; ++i)
      files[1 + i] = &pixB[i];
    unsigned long long wordTotal = 0, recTotal = 0;
    for (int i = 0; i <= kPixFiles; ++i) {
      mf.wordOff[i] = wordTotal;
      mf.recOff[i] = recTotal;
      mf.bytes[i] = files[i]->size();
      const unsigned long long w = files[i]->size() / 4;
      wordTotal += w;
      recTotal += w / 2;
    }
    mf.wordOff[1 + kPixFiles] = wordTotal;
    mf.recOff[1 + kPixFiles] = recTotal;
    std::vector<unsigned int> words(wordTotal);
    for (int i = 0; i <= kPixFiles; ++i)
      if (files[i]->size() >= 4)
        std::memcpy(words.data() + mf.wordOff[i], files[i]->data(), (files[i]->size() / 4) * 4);

    cudaError_t err = cudaSetDevice(device);
    Pool pool;
    Status* st = pool.get<Status>(1, err);
    unsigned int* dKeys = pool.get<unsigned int>(nMod, err);
    unsigned int* dSorted = pool.get<unsigned int>(nMod, err);
    unsigned int* dSrc = pool.get<unsigned int>(nMod, err);
    unsigned int* dCent = pool.get<unsigned int>(cent.size(), err);
    float* dEta = pool.get<float>(nSens, err);
    unsigned int* dEnd = pool.get<unsigned int>(size_t(nEnd) * 3, err);
    unsigned int* dTilt = pool.get<unsigned int>(size_t(nTilt) * 3, err);
    uint8_t* dEndLast = pool.get<uint8_t>(nEnd, err);
    uint8_t* dTiltLast = pool.get<uint8_t>(nTilt, err);
    unsigned int* dWords = pool.get<unsigned int>(wordTotal, err);
    mf.words = dWords;
    mf.recKey = pool.get<unsigned int>(recTotal, err);
    mf.recN = pool.get<unsigned int>(recTotal, err);
    mf.recStart = pool.get<unsigned long long>(recTotal, err);
    ModuleOut o{};
    o.detIds = pool.get<unsigned int>(nMod, err);
    o.layers = pool.get<short>(nMod, err);
    o.rings = pool.get<short>(nMod, err);
    o.modules = pool.get<short>(nMod, err);
    o.rods = pool.get<short>(nMod, err);
    o.subdets = pool.get<short>(nMod, err);
    o.sides = pool.get<short>(nMod, err);
    o.eta = pool.get<float>(nMod, err);
    o.r = pool.get<float>(nMod, err);
    o.isInverted = pool.get<uint8_t>(nMod, err);
    o.isLower = pool.get<uint8_t>(nMod, err);
    o.isAnchor = pool.get<uint8_t>(nMod, err);
    o.moduleType = pool.get<uint8_t>(nMod, err);
    o.moduleLayerType = pool.get<uint8_t>(nMod, err);
    o.sdlLayers = pool.get<int>(nMod, err);
    o.mapdetId = pool.get<unsigned int>(nMod, err);
    o.mapIdx = pool.get<uint16_t>(nMod, err);
    const size_t hashSize = size_t(1) << bits;
    unsigned int* dHashKey = pool.get<unsigned int>(hashSize, err);
    uint16_t* dHashVal = pool.get<uint16_t>(hashSize, err);
    unsigned int* dEndRecOf = pool.get<unsigned int>(nMod, err);
    unsigned int* dTiltRecOf = pool.get<unsigned int>(nMod, err);
    unsigned int* dGeoDetId = pool.get<unsigned int>(nEnd, err);
    float* dGeoPhi = pool.get<float>(nEnd, err);
    int* dGeoIndex = pool.get<int>(nMod, err);
    float* dDxdy = pool.get<float>(nMod, err);
    float* dDrdz = pool.get<float>(nMod, err);
    uint16_t* dPartner = pool.get<uint16_t>(nMod, err);
    unsigned int* dConnWin = pool.get<unsigned int>(nMod, err);
    unsigned int* dConnErr = pool.get<unsigned int>(nMod, err);
    uint16_t* dNConn = pool.get<uint16_t>(nMod, err);
    uint16_t* dModuleMap = pool.get<uint16_t>(size_t(nMod) * kMaxConnectedModules, err);
    unsigned int* dKeyRec = pool.get<unsigned int>(size_t(kPixFiles) * kPixKeys, err);
    unsigned int* dPixSizes = pool.get<unsigned int>(3 * size_t(kSizeSuperbins), err);
    unsigned int* dPixIndex = pool.get<unsigned int>(3 * size_t(kSizeSuperbins), err);
    const unsigned long long pixCapacity = std::max<unsigned long long>(wordTotal, 1);
    unsigned int* dPix = pool.get<unsigned int>(pixCapacity, err);
    int* dMdOffset = pool.get<int>(nLower + 1, err);
    int* dMdCap = pool.get<int>(nLower + 1, err);
    int* dLsOffset = pool.get<int>(nLower + 1, err);
    int* dLsCap = pool.get<int>(nLower + 1, err);
    int* dT3Cap = pool.get<int>(std::max(nLower, 1u), err);
    int* dT5Cap = pool.get<int>(std::max(nLower, 1u), err);
    auto cudaMsg = [&]() { return std::string("device event-setup build: ") + cudaGetErrorString(err); };
    if (err != cudaSuccess)
      return cudaMsg();

    auto up = [&](void* d, const void* h, size_t n) {
      if (err == cudaSuccess && n)
        err = cudaMemcpy(d, h, n, cudaMemcpyHostToDevice);
    };
    auto zero = [&](void* d, int v, size_t n) {
      if (err == cudaSuccess && n)
        err = cudaMemset(d, v, n);
    };
    up(dKeys, keys.data(), size_t(nMod) * 4);
    up(dCent, cent.data(), cent.size() * 4);
    up(dEta, etaRec.data(), size_t(nSens) * 4);
    up(dEnd, endB.data(), size_t(nEnd) * 12);
    up(dTilt, tiltB.data(), size_t(nTilt) * 12);
    up(dWords, words.data(), wordTotal * 4);
    Status init{};
    init.partnerMissing = kNone;
    init.connBad = kNone;
    init.pixSizeBad = kNone;
    init.pixUnknown = ~0ull;
    up(st, &init, sizeof(Status));
    // the host loader's defaults: zero, -1 for "none", 0xffff for an empty hash slot
    for (void* a : {static_cast<void*>(o.layers), static_cast<void*>(o.rings), static_cast<void*>(o.modules),
                    static_cast<void*>(o.rods), static_cast<void*>(o.subdets), static_cast<void*>(o.sides),
                    static_cast<void*>(dPartner), static_cast<void*>(dNConn)})
      zero(a, 0, size_t(nMod) * 2);
    for (void* a : {static_cast<void*>(o.eta), static_cast<void*>(o.r), static_cast<void*>(o.sdlLayers),
                    static_cast<void*>(o.detIds), static_cast<void*>(dConnWin)})
      zero(a, 0, size_t(nMod) * 4);
    for (void* a : {static_cast<void*>(o.isInverted), static_cast<void*>(o.isLower), static_cast<void*>(o.isAnchor),
                    static_cast<void*>(o.moduleType), static_cast<void*>(o.moduleLayerType)})
      zero(a, 0, nMod);
    for (void* a : {static_cast<void*>(dEndRecOf), static_cast<void*>(dTiltRecOf), static_cast<void*>(dGeoIndex)})
      zero(a, 0xff, size_t(nMod) * 4);
    zero(dHashKey, 0, hashSize * 4);
    zero(dHashVal, 0xff, hashSize * 2);
    zero(dModuleMap, 0, size_t(nMod) * kMaxConnectedModules * 2);
    zero(dKeyRec, 0, size_t(kPixFiles) * kPixKeys * 4);
    zero(dPix, 0, pixCapacity * 4);
    if (err != cudaSuccess)
      return cudaMsg();

    auto blocks = [](unsigned long long n, unsigned int t) {
      return static_cast<unsigned int>(std::max<unsigned long long>(1, (n + t - 1) / t));
    };
    auto status = [&]() {
      Status h{};
      if (err == cudaSuccess)
        err = cudaGetLastError();
      if (err == cudaSuccess)
        err = cudaMemcpy(&h, st, sizeof(Status), cudaMemcpyDeviceToHost);
      return h;
    };

    // detIds in ascending order; a duplicate among the sensors, then the
    // reserved detId, then the count, as the host loader checks them
    kRank<<<blocks(reserved ? nSens : nMod, 256), 256>>>(dKeys, reserved ? nSens : nMod, dSorted, dSrc, st);
    Status h = status();
    if (err != cudaSuccess)
      return cudaMsg();
    if (h.dup)
      return "duplicate detIds in sensor_centroids.bin";
    if (nMod > 65535)
      return "too many modules";
    if (reserved)
      return "detId 1 is reserved for the pixel module";
    kModules<<<1, 1024>>>(dSorted, dSrc, dCent, dEta, nMod, nLower, o, st);
    h = status();
    if (err != cudaSuccess)
      return cudaMsg();
    if (h.nLower > nLower)
      return "more lower modules than half of the sensors";
    if (h.nLower < nLower)
      return "module index out of range";
    kHash<<<1, 1>>>(o.mapdetId, o.mapIdx, nMod, bits, dHashKey, dHashVal);
    // orientations, then partners
    if (nEnd) {
      kLastOfKey<<<blocks(nEnd, 256), 256>>>(dEnd, nEnd, 3, dEndLast);
      kOrientIndex<<<blocks(nEnd, 256), 256>>>(dEnd, nEnd, dEndLast, true, dHashKey, dHashVal, bits, dEndRecOf,
                                               dGeoDetId, dGeoPhi, dGeoIndex, st);
    }
    if (nTilt) {
      kLastOfKey<<<blocks(nTilt, 256), 256>>>(dTilt, nTilt, 3, dTiltLast);
      kOrientIndex<<<blocks(nTilt, 256), 256>>>(dTilt, nTilt, dTiltLast, false, dHashKey, dHashVal, bits,
                                                dTiltRecOf, nullptr, nullptr, nullptr, st);
    }
    kOrientApply<<<blocks(nMod, 256), 256>>>(dEnd, dTilt, dEndRecOf, dTiltRecOf, o.detIds, o.subdets, nMod, dDxdy,
                                             dDrdz);
    kPartners<<<1, 1>>>(o.mapdetId, o.mapIdx, nMod, dHashKey, dHashVal, bits, o.isLower, o.isInverted, dPartner,
                        dDrdz, dDxdy, st);
    h = status();
    if (err != cudaSuccess)
      return cudaMsg();
    if (h.partnerMissing != kNone)
      return "partner sensor missing for detId " + std::to_string(h.partnerMissing);
    if (!pixMissing.empty())
      return pixMissing;

    // the map files: framing, the pixel map, then the connection map
    kFrame<<<1, 32>>>(mf, st);
    kPixWin<<<dim3(blocks(wordTotal / 2 + 1, 256), kPixFiles), 256>>>(mf, st, dKeyRec);
    kPixSizes<<<dim3(blocks(kSizeSuperbins, 256), 3), 256>>>(mf, dKeyRec, dPixSizes, st);
    kPixScan<<<3, 1024>>>(dPixSizes, dPixIndex, st);
    h = status();
    if (err != cudaSuccess)
      return cudaMsg();
    if (h.pixSizeBad != kNone)
      return "pixel map lists more than " + std::to_string(kMaxConnectedModules) + " modules for superbin " +
             std::to_string(h.pixSizeBad / 3);
    const unsigned long long nPixels = 0ull + h.pixTotal[0] + h.pixTotal[1] + h.pixTotal[2];
    if (nPixels > pixCapacity)
      return "pixel map larger than its files";
    kPixFill<<<dim3(blocks(kSizeSuperbins, 128), 3), 128>>>(mf, dKeyRec, dPixIndex, dHashKey, dHashVal, bits, dPix,
                                                            pixCapacity, st);
    h = status();
    if (err != cudaSuccess)
      return cudaMsg();
    if (h.pixUnknown != ~0ull)
      return "pixel map references an unknown detId " + std::to_string(h.pixUnknown & 0xffffffffull);
    kConnWin<<<blocks(mf.recOff[1] + 1, 256), 256>>>(mf, st, dHashKey, dHashVal, bits, dConnWin);
    kConnApply<<<blocks(nMod, 128), 128>>>(mf, dConnWin, o.detIds, nMod, dHashKey, dHashVal, bits, dNConn,
                                           dModuleMap, dConnErr, st);
    h = status();
    if (err != cudaSuccess)
      return cudaMsg();
    if (h.connBad != kNone) {
      // the first bad module in detId order, and what is wrong with it
      std::vector<unsigned int> detIds, detail;
      err = down(detIds, o.detIds, nMod);
      if (err == cudaSuccess)
        err = down(detail, dConnErr, nMod);
      if (err != cudaSuccess)
        return cudaMsg();
      const size_t i = std::find(detIds.begin(), detIds.end(), h.connBad) - detIds.begin();
      if (i < detail.size() && detail[i] != kNone)
        return "module map references an unknown detId " + std::to_string(detail[i]);
      return "more than " + std::to_string(kMaxConnectedModules) + " connected modules for detId " +
             std::to_string(h.connBad);
    }

    kCaps<<<1, 1024>>>(o.layers, o.subdets, o.rings, o.eta, dNConn, nLower, dMdOffset, dMdCap, dLsOffset, dLsCap,
                       dT3Cap, dT5Cap, st);
    h = status();
    if (err != cudaSuccess)
      return cudaMsg();

    // the host mirror
    es.nModules = static_cast<uint16_t>(nMod);
    es.nLowerModules = static_cast<uint16_t>(nLower);
    es.pixelModuleIndex = static_cast<uint16_t>(nLower);
    std::vector<unsigned int> index, sizes;
    cudaError_t e = cudaSuccess;
    auto get = [&](auto& v, const auto* d, size_t n) {
      if (e == cudaSuccess)
        e = down(v, d, n);
    };
    get(es.detIds, o.detIds, nMod);
    get(es.moduleMap, dModuleMap, size_t(nMod) * kMaxConnectedModules);
    get(es.nConnectedModules, dNConn, nMod);
    get(es.mapdetId, o.mapdetId, nMod);
    get(es.mapIdx, o.mapIdx, nMod);
    get(es.drdzs, dDrdz, nMod);
    get(es.dxdys, dDxdy, nMod);
    get(es.eta, o.eta, nMod);
    get(es.r, o.r, nMod);
    get(es.partnerModuleIndices, dPartner, nMod);
    get(es.layers, o.layers, nMod);
    get(es.rings, o.rings, nMod);
    get(es.modules, o.modules, nMod);
    get(es.rods, o.rods, nMod);
    get(es.subdets, o.subdets, nMod);
    get(es.sides, o.sides, nMod);
    get(es.isInverted, o.isInverted, nMod);
    get(es.isLower, o.isLower, nMod);
    get(es.isAnchor, o.isAnchor, nMod);
    get(es.moduleType, o.moduleType, nMod);
    get(es.moduleLayerType, o.moduleLayerType, nMod);
    get(es.sdlLayers, o.sdlLayers, nMod);
    get(es.connectedPixels, dPix, nPixels);
    get(index, dPixIndex, 3 * size_t(kSizeSuperbins));
    get(sizes, dPixSizes, 3 * size_t(kSizeSuperbins));
    get(es.geoMapDetId, dGeoDetId, h.geoCount);
    get(es.geoMapPhi, dGeoPhi, h.geoCount);
    get(es.geoMapIndex, dGeoIndex, nMod);
    get(es.mdOffset, dMdOffset, nLower + 1);
    get(es.mdCap, dMdCap, nLower + 1);
    get(es.lsOffset, dLsOffset, nLower + 1);
    get(es.lsCap, dLsCap, nLower + 1);
    get(es.t3CapIfUsed, dT3Cap, nLower);
    get(es.t5CapIfEligible, dT5Cap, nLower);
    get(es.detHashKey, dHashKey, hashSize);
    get(es.detHashVal, dHashVal, hashSize);
    if (e != cudaSuccess) {
      err = e;
      return cudaMsg();
    }
    es.detHashBits = bits;
    auto part = [&](int c, std::vector<unsigned int>& iv, std::vector<unsigned int>& sv) {
      iv.assign(index.begin() + size_t(c) * kSizeSuperbins, index.begin() + size_t(c + 1) * kSizeSuperbins);
      sv.assign(sizes.begin() + size_t(c) * kSizeSuperbins, sizes.begin() + size_t(c + 1) * kSizeSuperbins);
    };
    part(0, es.connectedPixelsIndex, es.connectedPixelsSizes);
    part(1, es.connectedPixelsIndexPos, es.connectedPixelsSizesPos);
    part(2, es.connectedPixelsIndexNeg, es.connectedPixelsSizesNeg);
    es.nPixels = static_cast<unsigned int>(nPixels);
    es.nTotalMDs = static_cast<unsigned int>(h.mdTotal) + kMaxPixelMDs;
    es.nTotalSegments = static_cast<unsigned int>(h.lsTotal) + kMaxPixelSegments;
    es.maxTriplets = h.t3Total;
    es.maxQuintuplets = h.t5Total;
    return std::string();
  }

}  // namespace lst
