// CUDA kernels of the LST object-building chain.  Every kernel takes the
// device event setup by value and an array of per-event views; blockIdx.y
// selects the event, so one launch processes a whole batch of events.
//
// Ordering.  The reference appends objects with atomic counters; its serial
// CPU backend therefore stores them in loop-nest order, and per-module
// occupancy caps keep the first N in that order.  Here each module (or pixel
// seed) is owned by one warp that walks the flattened loop nest in order,
// 32 candidates at a time, and places accepted objects with a warp ballot
// prefix, so object indices equal the reference CPU backend's.
#pragma once

#include <cuda_runtime.h>

#include "lst_device.h"

namespace lst {

  constexpr unsigned int kFullMask = 0xffffffffu;

  // T5 classifier weights (uploaded once per process from the weight file).
  __constant__ T5DnnWeights c_t5dnn;
  __constant__ float c_t5dnnWP = kT5DnnWP;  // DNN working point of the loaded weights

  struct ConstDnn {
    __device__ __forceinline__ const T5DnnWeights& get() const { return c_t5dnn; }
  };

  __device__ __forceinline__ unsigned int laneId() { return threadIdx.x & 31u; }
  __device__ __forceinline__ unsigned int lanesBelowMask() { return (1u << laneId()) - 1u; }

  // Rank of this lane's flag among the set flags of lower lanes; total = set flags in the warp.
  __device__ __forceinline__ unsigned int warpRank(bool flag, unsigned int& total) {
    unsigned int b = __ballot_sync(kFullMask, flag);
    total = __popc(b);
    return __popc(b & lanesBelowMask());
  }

  // Exclusive prefix sums of countOf(0..n-1) into pre[0..n] (pre[n] = total),
  // computed by one warp.  pre must be warp-private shared memory.
  template <typename F>
  __device__ __forceinline__ unsigned int warpPrefix(unsigned int* pre, int n, F countOf) {
    unsigned int carry = 0;
    for (int base = 0; base < n; base += 32) {
      int i = base + int(laneId());
      unsigned int c = (i < n) ? countOf(i) : 0u;
      unsigned int incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        unsigned int y = __shfl_up_sync(kFullMask, incl, o);
        if (int(laneId()) >= o)
          incl += y;
      }
      if (i < n)
        pre[i] = carry + incl - c;
      carry += __shfl_sync(kFullMask, incl, 31);
    }
    if (laneId() == 0)
      pre[n] = carry;
    __syncwarp();
    return carry;
  }

  // Largest k in [0, n) with pre[k] <= f (pre[n] > f).
  __device__ __forceinline__ int findSlot(const unsigned int* pre, int n, unsigned int f) {
    int lo = 0, hi = n;
    while (hi - lo > 1) {
      int mid = (lo + hi) >> 1;
      if (pre[mid] <= f)
        lo = mid;
      else
        hi = mid;
    }
    return lo;
  }

  // Block-wide exclusive scan (blockDim.x a multiple of 32, <= 1024).
  __device__ __forceinline__ unsigned int blockExclusiveScan(unsigned int v, unsigned int& total) {
    __shared__ unsigned int sWarp[32];
    __shared__ unsigned int sTotal;
    unsigned int lane = laneId(), wid = threadIdx.x >> 5;
    unsigned int nw = blockDim.x >> 5;
    unsigned int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      unsigned int y = __shfl_up_sync(kFullMask, incl, o);
      if (int(lane) >= o)
        incl += y;
    }
    if (lane == 31)
      sWarp[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      unsigned int w = (lane < nw) ? sWarp[lane] : 0u;
      unsigned int wi = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        unsigned int y = __shfl_up_sync(kFullMask, wi, o);
        if (int(lane) >= o)
          wi += y;
      }
      if (lane < nw)
        sWarp[lane] = wi - w;
      if (lane == 31)
        sTotal = wi;
    }
    __syncthreads();
    unsigned int excl = sWarp[wid] + incl - v;
    total = sTotal;
    __syncthreads();
    return excl;
  }

  // =============================================================== reset
  // Hit -> pLS index of the pLS cleaning: chains of (pLS, hit slot) entries
  // e = 4 pLS + slot in a hash table keyed by the stored pixel hit
  // (pLSHitsIdxs[e]): a head per bucket, a next entry per entry.  kPLSHitReset
  // empties the heads right before kPixelIngest inserts every entry once.
  constexpr unsigned int kPLSHitBucketBits = 15;
  constexpr unsigned int kPLSHitBuckets = 1u << kPLSHitBucketBits;
  constexpr unsigned int kPLSHitNone = 0xffffffffu;
  LST_DEV unsigned int plsHitBucket(unsigned int h) { return (h * 2654435761u) >> (32 - kPLSHitBucketBits); }

  __global__ void kPLSHitReset(const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    for (unsigned int i = blockIdx.x * blockDim.x + threadIdx.x; i < kPLSHitBuckets; i += gridDim.x * blockDim.x)
      ev.plsHitHead[i] = kPLSHitNone;
  }

  __global__ void kResetEvent(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned int nMod = es.nModules, nLower = es.nLowerModules;
    for (unsigned int i = blockIdx.x * blockDim.x + threadIdx.x; i < 2u * nMod; i += gridDim.x * blockDim.x) {
      ev.hits.hitRanges[i] = -1;
      ev.rg.mdRanges[i] = -1;
      ev.rg.segmentRanges[i] = -1;
      ev.rg.tripletRanges[i] = -1;
      ev.rg.quintupletRanges[i] = -1;
      if (i < nMod) {
        ev.hits.hitRangesLower[i] = -1;
        ev.hits.hitRangesUpper[i] = -1;
        ev.hits.hitRangesnLower[i] = -1;
        ev.hits.hitRangesnUpper[i] = -1;
      }
      if (i <= nLower) {
        ev.md.nMDs[i] = 0;
        ev.md.totOccupancyMDs[i] = 0;
        ev.ls.nSegments[i] = 0;
        ev.ls.totOccupancySegments[i] = 0;
        ev.rg.miniDoubletModuleIndices[i] = es.mdOffset[i];
        ev.rg.miniDoubletModuleOccupancy[i] = es.mdCap[i];
        ev.rg.segmentModuleIndices[i] = es.lsOffset[i];
        ev.rg.segmentModuleOccupancy[i] = es.lsCap[i];
      }
      if (i < nLower) {
        ev.t3.nTriplets[i] = 0;
        ev.t3.totOccupancyTriplets[i] = 0;
        ev.t5.nQuintuplets[i] = 0;
        ev.t5.totOccupancyQuintuplets[i] = 0;
        ev.rg.quintupletModuleIndices[i] = -1;
        ev.rg.quintupletModuleOccupancy[i] = 0;
        ev.rg.tripletModuleIndices[i] = 0;
        ev.rg.tripletModuleOccupancy[i] = 0;
      }
      if (i == 0) {
        ev.sc->status = 0;
        ev.sc->nPT5Total = 0;
        ev.sc->nPT3Total = 0;
        *ev.pt3.nPixelTriplets = 0;
        *ev.pt3.totOccupancyPixelTriplets = 0;
        *ev.pt5.nPixelQuintuplets = 0;
        *ev.pt5.totOccupancyPixelQuintuplets = 0;
        *ev.tc.nTrackCandidates = 0;
        *ev.tc.nTrackCandidatespT3 = 0;
        *ev.tc.nTrackCandidatespT5 = 0;
        *ev.tc.nTrackCandidatespLS = 0;
        *ev.tc.nTrackCandidatesT5 = 0;
        *ev.rg.nEligibleT5Modules = 0;
        *ev.rg.device_nTotalMDs = es.mdOffset[nLower];
        *ev.rg.device_nTotalSegs = es.lsOffset[nLower];
        *ev.rg.device_nTotalTrips = 0;
        *ev.rg.device_nTotalQuints = 0;
      }
    }
  }

  // ================================================================ hits
  // SDL/Hit.h:217-269
  __global__ void __launch_bounds__(256, 4) kHitPrep(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned int nHits = ev.sc->nHits;
    const Modules& m = es.m;
    Hits h = ev.hits;
    for (unsigned int ihit = blockIdx.x * blockDim.x + threadIdx.x; ihit < nHits; ihit += gridDim.x * blockDim.x) {
      float x = h.xs[ihit], y = h.ys[ihit], z = h.zs[ihit];
      unsigned int detId = h.detid[ihit];
      float rt = fsqrt(x * x + y * y);
      h.rts[ihit] = rt;
      h.phis[ihit] = phiOf(x, y);
      h.etas[ihit] = ((z > 0) - (z < 0)) * facosh(fsqrt(x * x + y * y + z * z) / rt);
      float hex = 0.f, hey = 0.f, lex = 0.f, ley = 0.f;
      int mIdx = -1;  // module of detId: the ES hash (linear probing)
      {
        const unsigned int mask = (1u << es.detHashBits) - 1;
        unsigned int slot = (detId * 2654435761u) >> (32 - es.detHashBits);
        for (unsigned int probe = 0; probe <= mask; ++probe) {
          const uint16_t val = es.detHashVal[slot];
          if (val == 0xffff)
            break;
          if (es.detHashKey[slot] == detId) {
            mIdx = val;
            break;
          }
          slot = (slot + 1) & mask;
        }
      }
      if (mIdx < 0) {
        atomicOr(&ev.sc->status, kStatusUnknownDetId);
        h.moduleIndices[ihit] = 0xffff;
        h.highEdgeXs[ihit] = hex;
        h.highEdgeYs[ihit] = hey;
        h.lowEdgeXs[ihit] = lex;
        h.lowEdgeYs[ihit] = ley;
        continue;
      }
      uint16_t mi = static_cast<uint16_t>(mIdx);
      h.moduleIndices[ihit] = mi;
      // Per-hit parts of the mini-doublet cuts of the module pair this hit
      // belongs to (lower module lm): the dphi-threshold slope, and the strip
      // shift of the hit it moves (tilted barrel and endcap modules).
      ev.hitMiniSlope[ihit] = mdMiniSlope(rt, m.ptCut);
      if (mi != es.pixelModule) {
        const bool isLowerHit = m.isLower[mi];
        const uint16_t lm = isLowerHit ? mi : m.partnerModuleIndices[mi];
        const bool shifted = m.subdets[lm] == Endcap || (m.subdets[lm] == Barrel && m.sides[lm] != Center);
        if (shifted && shiftMovesLower(m, lm) == isLowerHit) {
          float xa, ya, zn;
          shiftStripPrep(m, lm, x, y, z, rt, xa, ya, zn);
          ev.hitShiftXa[ihit] = xa;
          ev.hitShiftYa[ihit] = ya;
          ev.hitShiftZn[ihit] = zn;
        }
      }
      if (m.subdets[mi] == Endcap && m.moduleType[mi] == TwoS) {
        const int f = m.geoMapIndex[mi];  // sortedFind(m.geoMapDetId, detId, m.nEndCapMap), per module
        if (f < 0) {
          atomicOr(&ev.sc->status, kStatusUnknownEndcapDetId);
        } else {
          float phi = m.geoMapPhi[f];
          float cos_phi = fcos(phi);
          hex = x + 2.5f * cos_phi;
          lex = x - 2.5f * cos_phi;
          float sin_phi = fsin(phi);
          hey = y + 2.5f * sin_phi;
          ley = y - 2.5f * sin_phi;
        }
      }
      h.highEdgeXs[ihit] = hex;
      h.highEdgeYs[ihit] = hey;
      h.lowEdgeXs[ihit] = lex;
      h.lowEdgeYs[ihit] = ley;
      // The module's hit range [first, last]: the lanes of this warp on the
      // same module combine first, and one lane per module updates it.  The
      // first index starts at -1, the largest value as unsigned, so an
      // unsigned minimum takes the place of the reference's set-or-minimum.
      const unsigned int peers = __match_any_sync(__activemask(), static_cast<unsigned int>(mi));
      const unsigned int first = __reduce_min_sync(peers, ihit), last = __reduce_max_sync(peers, ihit);
      if (static_cast<unsigned int>(__ffs(peers) - 1) == (threadIdx.x & 31u)) {
        atomicMin(reinterpret_cast<unsigned int*>(&h.hitRanges[mi * 2]), first);
        atomicMax(&h.hitRanges[mi * 2 + 1], static_cast<int>(last));
      }
    }
  }

  // SDL/Hit.h:194-215
  __global__ void kModuleRanges(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    Hits h = ev.hits;
    for (unsigned int lower = blockIdx.x * blockDim.x + threadIdx.x; lower < es.nLowerModules;
         lower += gridDim.x * blockDim.x) {
      uint16_t upper = es.m.partnerModuleIndices[lower];
      if (h.hitRanges[lower * 2] != -1 && h.hitRanges[upper * 2] != -1) {
        h.hitRangesLower[lower] = h.hitRanges[lower * 2];
        h.hitRangesUpper[lower] = h.hitRanges[upper * 2];
        h.hitRangesnLower[lower] = static_cast<int8_t>(h.hitRanges[lower * 2 + 1] - h.hitRanges[lower * 2] + 1);
        h.hitRangesnUpper[lower] = static_cast<int8_t>(h.hitRanges[upper * 2 + 1] - h.hitRanges[upper * 2] + 1);
      }
    }
  }

  // ========================================================= pixel segments
  // SDL/Segment.h:1031-1117
  // Register budget: four 256-thread blocks per SM (at 154 registers a thread
  // only one fitted, and the kernel waits on gathers).
  __global__ void __launch_bounds__(256, 4) kPixelIngest(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned int nPLS = ev.sc->nPLS;
    const uint16_t pix = es.pixelModule;
    MiniDoublets md = ev.md;
    Segments ls = ev.ls;
    const unsigned int mdBase = es.mdOffset[es.nLowerModules];
    const unsigned int lsBase = es.lsOffset[es.nLowerModules];
    const unsigned int nHits = ev.sc->nHits;
    for (unsigned int tid = blockIdx.x * blockDim.x + threadIdx.x; tid < nPLS; tid += gridDim.x * blockDim.x) {
      unsigned int hit[4] = {ev.plsHit0[tid], ev.plsHit1[tid], ev.plsHit2[tid], ev.plsHit3[tid]};
      // The reference indexes the hit store with these unchecked; an index
      // outside the event is flagged and replaced by hit 0 (the host rejects
      // pixel segments for events without hits).
      for (int k = 0; k < 4; ++k)
        if (hit[k] >= nHits) {
          atomicOr(&ev.sc->status, kStatusInvalidInput);
          hit[k] = 0;
        }
      storePixelSegment(
          es.m, ev.hits, md, ls, pix, mdBase, lsBase, tid, hit[0], hit[1], hit[2], hit[3], ev.plsDPhiChange[tid]);
      ls.partOfPT5[tid] = 0;
      for (unsigned int slot = 0; slot < 4; ++slot) {
        const unsigned int e = 4 * tid + slot;
        ev.plsHitNext[e] = atomicExch(&ev.plsHitHead[plsHitBucket(ls.pLSHitsIdxs[e])], e);
      }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      md.nMDs[pix] = 2 * nPLS;
      md.totOccupancyMDs[pix] = 2 * nPLS;
      ls.nSegments[pix] = nPLS;
      ls.totOccupancySegments[pix] = nPLS;
    }
  }

  // Work counters of the kernels whose warps take their next task from the
  // event's counter (kCreateMD, kCreateLS, kCreateT3), so that a warp that
  // drew light tasks takes more: the work per module is very uneven.  Zeroed
  // before each of those kernels runs.
  __global__ void kTaskCountersReset(const EventView* evs) {
    if (threadIdx.x == 0) {
      EventScalars* sc = evs[blockIdx.y].sc;
      sc->mdNext = 0;
      sc->lsNext = 0;
      sc->t3Next = 0;
    }
  }
  // The next task of the calling warp from counter *next (the same value on
  // every lane).
  __device__ __forceinline__ unsigned int warpNextTask(unsigned int* next) {
    unsigned int t = 0;
    if (laneId() == 0)
      t = atomicAdd(next, 1u);
    return __shfl_sync(kFullMask, t, 0);
  }

  // ======================================================== mini-doublets
  // SDL/MiniDoublet.h:896-992: every (lower hit, upper hit) pair of a lower
  // module is a candidate; passing ones are stored in the module's arena at
  // their rank in the reference's serial loop order (lower hit outer, upper
  // hit inner), the first mdCap of them.
  //
  // A warp takes up to 32 consecutive lower modules at a time (most hold
  // fewer than 32 pairs, the median 14) and deals their pairs out in order, 32
  // per step, across module boundaries: lane l of step s takes the task's pair
  // 32 s + l, finds its module by a binary search over the lanes' exclusive
  // prefix of pair counts, and its hits by dividing by the module's upper
  // hit count.  A passing pair's rank is the module's running count (one
  // word per module in shared memory) plus the passing lanes of the same
  // module below it (__match_any_sync).  So the lanes stay busy on small
  // modules, and a large module simply spans several steps.
  constexpr int kMDMaxWarps = 8;  // warps per block the kernel is launched with (at most)
  __device__ __forceinline__ void mdTask(DeviceES const& es, const EventView& ev, unsigned int task,
                                         unsigned int modulesPerTask, unsigned int* count) {
    const Hits& h = ev.hits;
    const unsigned int lane = laneId();
    const unsigned int lmU = task * modulesPerTask + lane;
    const bool valid = lane < modulesPerTask && lmU < es.nLowerModules && h.hitRangesLower[lmU] != -1;
    const int nL = valid ? int(h.hitRangesnLower[lmU]) : 0;
    const int nU = valid ? int(h.hitRangesnUpper[lmU]) : 0;
    const int loHit0 = valid ? h.hitRangesLower[lmU] : 0;
    const int upHit0 = valid ? h.hitRangesUpper[lmU] : 0;
    const int cap = valid ? es.mdCap[lmU] : 0;
    const unsigned int base = valid ? es.mdOffset[lmU] : 0u;
    // (the reference's counts are int8; a negative one means no pairs here)
    const int pairs = (nL > 0 && nU > 0) ? nL * nU : 0;
    int incl = pairs;  // inclusive prefix of the pair counts over the lanes
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int o = __shfl_up_sync(kFullMask, incl, d);
      if (int(lane) >= d)
        incl += o;
    }
    const int excl = incl - pairs;
    const int total = __shfl_sync(kFullMask, incl, 31);
    count[lane] = 0;
    __syncwarp();
    MiniDoublets md = ev.md;
    const MDHitPre pre{ev.hitMiniSlope, ev.hitShiftXa, ev.hitShiftYa, ev.hitShiftZn};
    for (int start = 0; start < total; start += 32) {
      const int g = start + int(lane);
      // the module of pair g: the last lane whose exclusive prefix is <= g
      // (a lane without pairs shares its prefix with the next one)
      int j = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const int e = __shfl_sync(kFullMask, excl, (j + step) & 31);
        if (j + step < 32 && e <= g)
          j += step;
      }
      const int exj = __shfl_sync(kFullMask, excl, j);
      const int nUj = __shfl_sync(kFullMask, nU, j);
      const int loj = __shfl_sync(kFullMask, loHit0, j);
      const int upj = __shfl_sync(kFullMask, upHit0, j);
      const int capj = __shfl_sync(kFullMask, cap, j);
      const unsigned int basej = __shfl_sync(kFullMask, base, j);
      bool ok = false;
      MDValues v;
      unsigned int lowerIdx = 0, upperIdx = 0;
      const uint16_t lm = static_cast<uint16_t>(task * modulesPerTask + unsigned(j));
      if (g < total) {
        const int local = g - exj;
        lowerIdx = unsigned(loj + local / nUj);
        upperIdx = unsigned(upj + local % nUj);
        ok = mdSelect(es.m, lm, h.xs[lowerIdx], h.ys[lowerIdx], h.zs[lowerIdx], h.rts[lowerIdx], h.xs[upperIdx],
                      h.ys[upperIdx], h.zs[upperIdx], h.rts[upperIdx], h.phis[lowerIdx], h.phis[upperIdx], pre,
                      lowerIdx, upperIdx, v);
      }
      const unsigned int peers = __match_any_sync(kFullMask, ok ? unsigned(j) : 32u + lane);
      const unsigned int rank = __popc(peers & lanesBelowMask());
      if (ok) {
        const unsigned int r = count[j] + rank;
        if (int(r) < capj)
          storeMD(es.m, h, md, lowerIdx, upperIdx, lm, v, basej + r);
      }
      __syncwarp();
      if (ok && rank == 0)
        count[j] += __popc(peers);
      __syncwarp();
    }
    if (valid) {
      const unsigned int n = count[lane];
      md.nMDs[lmU] = (int(n) < cap) ? n : (cap > 0 ? unsigned(cap) : 0u);
      md.totOccupancyMDs[lmU] = n;
      if (int(n) > cap)
        atomicOr(&ev.sc->status, kStatusCapOverflow);
    }
    __syncwarp();
  }

  // Register budgets of the cut kernels, as resident blocks per SM.  The cut
  // kernels wait mostly on dependent loads, so they run faster with more warps
  // resident even where the tighter budget spills a little; the values are
  // the fastest of a sweep over 2..14 blocks on B200 (PU200 batches, launch
  // shapes autotuned for each setting).
#ifndef LST_LB_MD_B
#define LST_LB_MD_B 4
#endif
#ifndef LST_LB_LS_B
#define LST_LB_LS_B 12
#endif
#ifndef LST_LB_T3_B
#define LST_LB_T3_B 10
#endif
#ifndef LST_LB_EVAL_B
#define LST_LB_EVAL_B 10
#endif
#ifndef LST_LB_T5EVAL_B
#define LST_LB_T5EVAL_B 8
#endif
#ifndef LST_LB_PIXMID_B
#define LST_LB_PIXMID_B 12
#endif
#define LST_LB_MD 256, LST_LB_MD_B
#define LST_LB_LS 128, LST_LB_LS_B
#define LST_LB_T3 128, LST_LB_T3_B
#define LST_LB_EVAL 128, LST_LB_EVAL_B
#define LST_LB_T5EVAL 128, LST_LB_T5EVAL_B
#define LST_LB_PIXMID 128, LST_LB_PIXMID_B
  // modulesPerTask (1..32): 8 for batches; fewer for a single event, whose
  // 13 000 lower modules would otherwise make only ~400 warp tasks.
  __global__ void __launch_bounds__(LST_LB_MD) kCreateMD(DeviceES es, const EventView* evs, unsigned int modulesPerTask) {
    __shared__ unsigned int sCount[kMDMaxWarps][32];
    const EventView& ev = evs[blockIdx.y];
    const int w = threadIdx.x >> 5;
    const unsigned int nTasks = (es.nLowerModules + modulesPerTask - 1u) / modulesPerTask;
    // tasks from the event's counter (kTaskCountersReset zeroes it before)
    for (unsigned int task = warpNextTask(&ev.sc->mdNext); task < nTasks; task = warpNextTask(&ev.sc->mdNext))
      mdTask(es, ev, task, modulesPerTask, sCount[w]);
  }

  // Derived per-MD values for every stored MD (lower modules and the pixel
  // module).  A warp takes 32 lower modules at a time (a module holds a few
  // MDs) and shares their MDs out over its lanes: a lane-level prefix of the
  // modules' counts, and per MD the owning lane by a search over it.
  // The pixel module's mini-doublets (two per pLS, thousands per event) are
  // shared out over all of the event's threads.
  __global__ void kMDDerived(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned int nWarps = gridDim.x * (blockDim.x >> 5);
    const unsigned int lane = laneId();
    MiniDoublets md = ev.md;
    for (unsigned int w0 = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32u; w0 < es.nLowerModules;
         w0 += nWarps * 32u) {
      const unsigned int w = w0 + lane;
      const unsigned int n = w < es.nLowerModules ? md.nMDs[w] : 0u;
      const unsigned int base = w < es.nLowerModules ? static_cast<unsigned int>(es.mdOffset[w]) : 0u;
      unsigned int incl = n;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned int y = __shfl_up_sync(kFullMask, incl, o);
        if (int(lane) >= o)
          incl += y;
      }
      const unsigned int total = __shfl_sync(kFullMask, incl, 31);
      for (unsigned int f0 = 0; f0 < total; f0 += 32) {
        const unsigned int f = f0 + lane;
        // owner: the first lane whose inclusive count exceeds f
        int owner = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
          const unsigned int c = __shfl_sync(kFullMask, incl, owner + step - 1);
          if (c <= f)
            owner += step;
        }
        const unsigned int ownerIncl = __shfl_sync(kFullMask, incl, owner);
        const unsigned int ownerN = __shfl_sync(kFullMask, n, owner);
        const unsigned int ownerBase = __shfl_sync(kFullMask, base, owner);
        if (f < total)
          storeMDDerived(md, ownerBase + (f - (ownerIncl - ownerN)), es.m.ptCut);
      }
    }
    const unsigned int nPix = md.nMDs[es.nLowerModules];
    const unsigned int pixBase = es.mdOffset[es.nLowerModules];
    for (unsigned int k = blockIdx.x * blockDim.x + threadIdx.x; k < nPix; k += gridDim.x * blockDim.x)
      storeMDDerived(md, pixBase + k, es.m.ptCut);
  }

  // SDL/MiniDoublet.h:1084-1104
  __global__ void kMDRanges(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    for (unsigned int i = blockIdx.x * blockDim.x + threadIdx.x; i < es.nLowerModules; i += gridDim.x * blockDim.x) {
      if (ev.md.nMDs[i] == 0 or ev.hits.hitRanges[i * 2] == -1) {
        ev.rg.mdRanges[i * 2] = -1;
        ev.rg.mdRanges[i * 2 + 1] = -1;
      } else {
        ev.rg.mdRanges[i * 2] = es.mdOffset[i];
        ev.rg.mdRanges[i * 2 + 1] = es.mdOffset[i] + ev.md.nMDs[i] - 1;
      }
    }
  }

  // ======================================================== line segments
  // One warp per inner lower module walking (connected module, inner MD,
  // outer MD) in order (SDL/Segment.h:798-910).
  constexpr int kLSWarps = 4;
  // Per-warp scratch of the walk: the prefix of the candidates over the
  // connected modules, and per connected module its index, MD count and
  // first MD, so that a candidate finds its MDs without a global load.
  struct LSScratch {
    unsigned int pre[kMaxConnectedModules + 1];
    unsigned int nOuterMDs[kMaxConnectedModules];
    unsigned int outerBase[kMaxConnectedModules];
    uint16_t outer[kMaxConnectedModules];
  };
  __device__ __forceinline__ void lsModule(DeviceES const& es, const EventView& ev, uint16_t lm, LSScratch& sc) {
    const unsigned int nInnerMDs = ev.md.nMDs[lm];
    if (nInnerMDs == 0)
      return;
    const Modules& m = es.m;
    const int nConn = m.nConnectedModules[lm];
    uint16_t* outer = sc.outer;
    const unsigned int total = warpPrefix(sc.pre, nConn, [&](int k) {
      const uint16_t o = m.moduleMap[lm * kMaxConnectedModules + k];
      const unsigned int n = ev.md.nMDs[o];
      outer[k] = o;
      sc.nOuterMDs[k] = n;
      sc.outerBase[k] = static_cast<unsigned int>(es.mdOffset[o]);
      return nInnerMDs * n;
    });
    const int cap = es.lsCap[lm];
    const unsigned int base = es.lsOffset[lm];
    const unsigned int innerBase = es.mdOffset[lm];
    Segments ls = ev.ls;
    unsigned int count = 0;
    for (unsigned int start = 0; start < total; start += 32) {
      unsigned int f = start + laneId();
      bool ok = false;
      LSValues v;
      unsigned int innerMD = 0, outerMD = 0;
      uint16_t outerLM = 0;
      if (f < total) {
        int k = findSlot(sc.pre, nConn, f);
        outerLM = outer[k];
        unsigned int nOuterMDs = sc.nOuterMDs[k];
        unsigned int local = f - sc.pre[k];
        innerMD = innerBase + local / nOuterMDs;
        outerMD = sc.outerBase[k] + local % nOuterMDs;
        ok = lsSelect(m, ev.md, lm, outerLM, innerMD, outerMD, v);
      }
      unsigned int tot;
      unsigned int r = count + warpRank(ok, tot);
      if (ok && int(r) < cap)
        storeLS(ls, ev.md, innerMD, outerMD, lm, outerLM, v, base + r);
      count += tot;
    }
    if (laneId() == 0) {
      ls.nSegments[lm] = (int(count) < cap) ? count : (cap > 0 ? unsigned(cap) : 0u);
      ls.totOccupancySegments[lm] = count;
      if (int(count) > cap)
        atomicOr(&ev.sc->status, kStatusCapOverflow);
    }
  }

  __global__ void __launch_bounds__(LST_LB_LS) kCreateLS(DeviceES es, const EventView* evs) {
    __shared__ LSScratch sScratch[kLSWarps];
    const EventView& ev = evs[blockIdx.y];
    const int wib = threadIdx.x >> 5;
    // modules from the event's counter (kTaskCountersReset zeroes it before)
    for (unsigned int w = warpNextTask(&ev.sc->lsNext); w < es.nLowerModules; w = warpNextTask(&ev.sc->lsNext)) {
      __syncwarp();
      lsModule(es, ev, static_cast<uint16_t>(w), sScratch[wib]);
    }
  }

  // SDL/Segment.h:1010-1029
  __global__ void kLSRanges(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    for (unsigned int i = blockIdx.x * blockDim.x + threadIdx.x; i < es.nLowerModules; i += gridDim.x * blockDim.x) {
      if (ev.ls.nSegments[i] == 0) {
        ev.rg.segmentRanges[i * 2] = -1;
        ev.rg.segmentRanges[i * 2 + 1] = -1;
      } else {
        ev.rg.segmentRanges[i * 2] = es.lsOffset[i];
        ev.rg.segmentRanges[i * 2 + 1] = es.lsOffset[i] + ev.ls.nSegments[i] - 1;
      }
    }
  }

  // ================================================= MD-keyed indices
  // For one module: the objects [0, n) of the module (segments or triplets,
  // in storage order) grouped by the module-local index of their first
  // mini-doublet, stably, so that each group keeps storage order.  Written:
  // start[md] / count[md] for every MD of the module, perm[] the object
  // indices (module-relative).  One warp; `bins` / `cursor` are warp-private
  // shared arrays of kMaxModuleMDs entries.
  constexpr int kMaxModuleMDs = 128;

  template <typename FirstMD>
  __device__ __forceinline__ void buildByMD(unsigned int n, unsigned int nBins, FirstMD firstMD, uint16_t* start,
                                            uint16_t* count, uint16_t* perm, unsigned int* bins,
                                            unsigned int* cursor) {
    for (unsigned int b = laneId(); b < nBins; b += 32)
      bins[b] = 0;
    __syncwarp();
    for (unsigned int k = laneId(); k < n; k += 32)
      atomicAdd(&bins[firstMD(k)], 1u);
    __syncwarp();
    // exclusive scan of the bins
    unsigned int carry = 0;
    for (unsigned int b0 = 0; b0 < nBins; b0 += 32) {
      unsigned int b = b0 + laneId();
      unsigned int c = b < nBins ? bins[b] : 0u;
      unsigned int incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        unsigned int y = __shfl_up_sync(kFullMask, incl, o);
        if (int(laneId()) >= o)
          incl += y;
      }
      if (b < nBins) {
        cursor[b] = carry + incl - c;
        start[b] = static_cast<uint16_t>(carry + incl - c);
        count[b] = static_cast<uint16_t>(c);
      }
      carry += __shfl_sync(kFullMask, incl, 31);
    }
    __syncwarp();
    // stable placement, 32 objects at a time
    for (unsigned int k0 = 0; k0 < n; k0 += 32) {
      unsigned int k = k0 + laneId();
      bool valid = k < n;
      unsigned int b = valid ? firstMD(k) : 0xffffffffu;
      unsigned int active = __ballot_sync(kFullMask, valid);
      unsigned int peers = __match_any_sync(kFullMask, b) & active;
      if (valid) {
        unsigned int rank = __popc(peers & lanesBelowMask());
        perm[cursor[b] + rank] = static_cast<uint16_t>(k);
      }
      __syncwarp();
      if (valid && laneId() == 31u - __clz(peers))
        cursor[b] += __popc(peers);
      __syncwarp();
    }
  }

  // The same grouping for 32 consecutive modules at once (most modules hold a
  // few objects): their bins lie side by side in bins[0, sum of the modules'
  // MDs), each object is counted into its module's bin, and a module-relative
  // start is the running count over all bins minus the objects of the
  // group's earlier modules (each object lies in a bin of its own module).
  // Placement takes the group's objects in storage order, so each group stays
  // stable.  The module of the f-th object or b-th bin is found by a search
  // over the lanes' prefix counts.  Returns false (having written nothing)
  // when the bins do not fit, and the caller groups module by module.
  // nOf(w) = objects of module w (0 for a module past the end), objBase(w) =
  // its first object, firstMD(w, k) = module-relative first MD of object k.
  constexpr unsigned int kByMDGroupBins = 512;
  constexpr int kByMDKeptChunks = 8;  // bins of the first chunks kept in registers between the passes
  __device__ __forceinline__ int laneOwner(unsigned int incl, unsigned int f) {
    int owner = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
      const unsigned int c = __shfl_sync(kFullMask, incl, owner + step - 1);
      if (c <= f)
        owner += step;
    }
    return owner;
  }
  __device__ __forceinline__ unsigned int laneInclusiveSum(unsigned int v) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned int y = __shfl_up_sync(kFullMask, v, o);
      if (int(laneId()) >= o)
        v += y;
    }
    return v;
  }

  template <typename NOf, typename ObjBase, typename FirstMD>
  __device__ __forceinline__ bool buildByMDGroup(DeviceES const& es, const EventView& ev, unsigned int w0, NOf nOf,
                                                 ObjBase objBase, FirstMD firstMD, uint16_t* start, uint16_t* count,
                                                 uint16_t* perm, unsigned int* bins, unsigned int* cursor) {
    const unsigned int lane = laneId();
    const unsigned int w = w0 + lane;
    const bool inRange = w < es.nLowerModules;
    const unsigned int n = inRange ? nOf(w) : 0u;
    const unsigned int nMD = (inRange && n > 0) ? ev.md.nMDs[w] : 0u;
    const unsigned int mdBase = inRange ? static_cast<unsigned int>(es.mdOffset[w]) : 0u;
    const unsigned int base = (inRange && n > 0) ? objBase(w) : 0u;
    const unsigned int objIncl = laneInclusiveSum(n), binIncl = laneInclusiveSum(nMD);
    const unsigned int nObj = __shfl_sync(kFullMask, objIncl, 31), nBins = __shfl_sync(kFullMask, binIncl, 31);
    if (nBins > kByMDGroupBins)
      return false;
    if (nObj == 0)
      return true;
    const unsigned int objExcl = objIncl - n, binExcl = binIncl - nMD;
    for (unsigned int b = lane; b < nBins; b += 32)
      bins[b] = 0;
    __syncwarp();
    unsigned int kept[kByMDKeptChunks];
    for (unsigned int f0 = 0; f0 < nObj; f0 += 32) {
      const unsigned int f = f0 + lane;
      const int o = laneOwner(objIncl, f);
      const unsigned int oObjExcl = __shfl_sync(kFullMask, objExcl, o);
      const unsigned int oBinExcl = __shfl_sync(kFullMask, binExcl, o);
      unsigned int bin = 0xffffffffu;
      if (f < nObj) {
        bin = oBinExcl + firstMD(w0 + o, f - oObjExcl);
        atomicAdd(&bins[bin], 1u);
      }
#pragma unroll
      for (int c = 0; c < kByMDKeptChunks; ++c)
        if (f0 == 32u * c)
          kept[c] = bin;
    }
    __syncwarp();
    // running count over all bins -> module-relative starts
    unsigned int carry = 0;
    for (unsigned int b0 = 0; b0 < nBins; b0 += 32) {
      const unsigned int b = b0 + lane;
      const unsigned int c = b < nBins ? bins[b] : 0u;
      const unsigned int incl = laneInclusiveSum(c);
      const int o = laneOwner(binIncl, b);
      const unsigned int oObjExcl = __shfl_sync(kFullMask, objExcl, o);
      const unsigned int oBinExcl = __shfl_sync(kFullMask, binExcl, o);
      const unsigned int oMdBase = __shfl_sync(kFullMask, mdBase, o);
      if (b < nBins) {
        const unsigned int rel = carry + incl - c - oObjExcl;
        cursor[b] = rel;
        start[oMdBase + (b - oBinExcl)] = static_cast<uint16_t>(rel);
        count[oMdBase + (b - oBinExcl)] = static_cast<uint16_t>(c);
      }
      carry += __shfl_sync(kFullMask, incl, 31);
    }
    __syncwarp();
    // stable placement, 32 objects at a time
    for (unsigned int f0 = 0; f0 < nObj; f0 += 32) {
      const unsigned int f = f0 + lane;
      const int o = laneOwner(objIncl, f);
      const unsigned int oObjExcl = __shfl_sync(kFullMask, objExcl, o);
      const unsigned int oBinExcl = __shfl_sync(kFullMask, binExcl, o);
      const unsigned int oBase = __shfl_sync(kFullMask, base, o);
      const bool valid = f < nObj;
      const unsigned int k = f - oObjExcl;
      unsigned int bin = 0xffffffffu;
      if (f0 < 32u * kByMDKeptChunks) {
#pragma unroll
        for (int c = 0; c < kByMDKeptChunks; ++c)
          if (f0 == 32u * c)
            bin = kept[c];
      } else if (valid) {
        bin = oBinExcl + firstMD(w0 + o, k);
      }
      const unsigned int active = __ballot_sync(kFullMask, valid);
      const unsigned int peers = __match_any_sync(kFullMask, bin) & active;
      if (valid) {
        const unsigned int rank = __popc(peers & lanesBelowMask());
        perm[oBase + cursor[bin] + rank] = static_cast<uint16_t>(k);
      }
      __syncwarp();
      if (valid && lane == 31u - __clz(peers))
        cursor[bin] += __popc(peers);
      __syncwarp();
    }
    return true;
  }

  // Segments of each lower module grouped by inner MD (after kCreateLS): a
  // warp takes 32 modules at a time, module by module where their bins do
  // not fit (or the fallback paths are forced).
  constexpr int kIdxWarps = 4;
  __global__ void kLSByMD(DeviceES es, const EventView* evs) {
    __shared__ unsigned int sBins[kIdxWarps][kByMDGroupBins];
    __shared__ unsigned int sCursor[kIdxWarps][kByMDGroupBins];
    const EventView& ev = evs[blockIdx.y];
    const int wib = threadIdx.x >> 5;
    const unsigned int* mdIdx = ev.ls.mdIndices;
    const unsigned int nWarps = gridDim.x * kIdxWarps;
    for (unsigned int w0 = (blockIdx.x * kIdxWarps + wib) * 32u; w0 < es.nLowerModules; w0 += nWarps * 32u) {
      __syncwarp();
      if (!ev.forceWalk &&
          buildByMDGroup(
              es, ev, w0, [&](unsigned int w) { return static_cast<unsigned int>(ev.ls.nSegments[w]); },
              [&](unsigned int w) { return static_cast<unsigned int>(es.lsOffset[w]); },
              [&](unsigned int w, unsigned int k) { return mdIdx[2 * (es.lsOffset[w] + k)] - es.mdOffset[w]; },
              ev.mdLSStart, ev.mdLSCount, ev.lsByMD, sBins[wib], sCursor[wib]))
        continue;
      for (unsigned int w = w0; w < w0 + 32u && w < es.nLowerModules; ++w) {
        __syncwarp();
        const unsigned int n = ev.ls.nSegments[w];
        if (n == 0)
          continue;
        const unsigned int mdBase = es.mdOffset[w];
        const unsigned int nMD = ev.md.nMDs[w];
        const unsigned int segBase = es.lsOffset[w];
        buildByMD(
            n, nMD, [&](unsigned int k) { return mdIdx[2 * (segBase + k)] - mdBase; }, ev.mdLSStart + mdBase,
            ev.mdLSCount + mdBase, ev.lsByMD + segBase, sBins[wib], sCursor[wib]);
      }
    }
  }

  // Triplets of each lower module grouped by first MD (after kCreateT3), in
  // the same way.
  __global__ void kT3ByMD(DeviceES es, const EventView* evs) {
    __shared__ unsigned int sBins[kIdxWarps][kByMDGroupBins];
    __shared__ unsigned int sCursor[kIdxWarps][kByMDGroupBins];
    const EventView& ev = evs[blockIdx.y];
    const int wib = threadIdx.x >> 5;
    const unsigned int* segIdx = ev.t3.segmentIndices;
    const unsigned int* mdIdx = ev.ls.mdIndices;
    const unsigned int nWarps = gridDim.x * kIdxWarps;
    for (unsigned int w0 = (blockIdx.x * kIdxWarps + wib) * 32u; w0 < es.nLowerModules; w0 += nWarps * 32u) {
      __syncwarp();
      if (!ev.forceWalk &&
          buildByMDGroup(
              es, ev, w0, [&](unsigned int w) { return static_cast<unsigned int>(ev.t3.nTriplets[w]); },
              [&](unsigned int w) { return static_cast<unsigned int>(ev.rg.tripletModuleIndices[w]); },
              [&](unsigned int w, unsigned int k) {
                return mdIdx[2 * segIdx[2 * (ev.rg.tripletModuleIndices[w] + k)]] - es.mdOffset[w];
              },
              ev.mdT3Start, ev.mdT3Count, ev.t3ByMD, sBins[wib], sCursor[wib]))
        continue;
      for (unsigned int w = w0; w < w0 + 32u && w < es.nLowerModules; ++w) {
        __syncwarp();
        const unsigned int n = ev.t3.nTriplets[w];
        if (n == 0)
          continue;
        const unsigned int mdBase = es.mdOffset[w];
        const unsigned int nMD = ev.md.nMDs[w];
        const unsigned int t3Base = ev.rg.tripletModuleIndices[w];
        buildByMD(
            n, nMD, [&](unsigned int k) { return mdIdx[2 * segIdx[2 * (t3Base + k)]] - mdBase; },
            ev.mdT3Start + mdBase, ev.mdT3Count + mdBase, ev.t3ByMD + t3Base, sBins[wib], sCursor[wib]);
      }
    }
  }

  // ============================================================ triplets
  // Per-module triplet offsets (SDL/Triplet.h:1007-1102); one block per event.
  __global__ void __launch_bounds__(1024) kT3Offsets(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    unsigned int carry = 0;
    for (unsigned int base = 0; base < es.nLowerModules; base += blockDim.x) {
      unsigned int i = base + threadIdx.x;
      unsigned int occ = 0;
      bool valid = i < es.nLowerModules;
      if (valid && ev.ls.nSegments[i] != 0)
        occ = static_cast<unsigned int>(es.t3CapIfUsed[i]);
      unsigned int tot;
      unsigned int ex = blockExclusiveScan(occ, tot);
      if (valid) {
        ev.rg.tripletModuleIndices[i] = static_cast<int>(carry + ex);
        ev.rg.tripletModuleOccupancy[i] = static_cast<int>(occ);
      }
      carry += tot;
    }
    if (threadIdx.x == 0)
      *ev.rg.device_nTotalTrips = carry;
  }

  // One warp per inner-inner lower module walking (inner segment, outer
  // segment of the middle module) in order (SDL/Triplet.h:874-1005).
  //
  // The inner segments are taken kT3Chunk at a time.  For each the warp
  // keeps in shared memory the prefix of its candidates and where its outer
  // segments are listed (the MD-keyed segment index of the middle module),
  // so that a candidate reaches its outer segment with one global load.
  constexpr int kT3Warps = 4;
  constexpr int kT3Chunk = 128;
  struct T3Scratch {
    unsigned int pre[kT3Chunk + 1];
    unsigned int listStart[kT3Chunk];  // first entry of the inner segment's outer segments in lsByMD
    unsigned int outerBase[kT3Chunk];  // first segment of the middle module
  };
  __device__ __forceinline__ void t3Module(DeviceES const& es, const EventView& ev, uint16_t lm1, T3Scratch& sc) {
    const Modules& m = es.m;
    if (m.nConnectedModules[lm1] == 0)
      return;
    const unsigned int nInner = ev.ls.nSegments[lm1];
    if (nInner == 0)
      return;
    const unsigned int segBase = es.lsOffset[lm1];
    const Segments& ls = ev.ls;
    const int cap = ev.rg.tripletModuleOccupancy[lm1];
    const unsigned int base = ev.rg.tripletModuleIndices[lm1];
    Triplets t3 = ev.t3;
    unsigned int count = 0;
    for (unsigned int c0 = 0; c0 < nInner; c0 += kT3Chunk) {
      const int n = int(min(nInner - c0, unsigned(kT3Chunk)));
      __syncwarp();  // the previous chunk's scratch has been read
      // Only outer segments whose inner MD is the inner segment's outer MD
      // can pass (the first test of the reference's triplet algorithm); they
      // are enumerated through the MD-keyed segment index in storage order,
      // so candidates keep the reference's (inner, outer) order.
      const unsigned int total = warpPrefix(sc.pre, n, [&](int i) {
        const unsigned int seg = segBase + c0 + unsigned(i);
        const uint16_t middle = ls.outerLowerModuleIndices[seg];
        if (ls.nSegments[middle] == 0)
          return 0u;
        const unsigned int mdMid = ls.mdIndices[2 * seg + 1];
        const unsigned int outerBase = es.lsOffset[middle];
        sc.outerBase[i] = outerBase;
        sc.listStart[i] = outerBase + ev.mdLSStart[mdMid];
        return static_cast<unsigned int>(ev.mdLSCount[mdMid]);
      });
      for (unsigned int start = 0; start < total; start += 32) {
        unsigned int f = start + laneId();
        bool ok = false;
        T3Values v;
        unsigned int innerSeg = 0, outerSeg = 0;
        uint16_t middle = 0, outerOuter = 0;
        if (f < total) {
          int i = findSlot(sc.pre, n, f);
          innerSeg = segBase + c0 + unsigned(i);
          middle = ls.outerLowerModuleIndices[innerSeg];
          outerSeg = sc.outerBase[i] + ev.lsByMD[sc.listStart[i] + (f - sc.pre[i])];
          outerOuter = ls.outerLowerModuleIndices[outerSeg];
          ok = t3Select(m, ev.md, ls, lm1, middle, outerOuter, innerSeg, outerSeg, v);
        }
        unsigned int tot;
        unsigned int r = count + warpRank(ok, tot);
        if (ok && int(r) < cap)
          storeT3(m, ev.md, ls, t3, innerSeg, outerSeg, lm1, middle, outerOuter, v, base + r);
        count += tot;
      }
    }
    if (laneId() == 0) {
      t3.nTriplets[lm1] = (int(count) < cap) ? count : (cap > 0 ? unsigned(cap) : 0u);
      t3.totOccupancyTriplets[lm1] = count;
      if (int(count) > cap)
        atomicOr(&ev.sc->status, kStatusCapOverflow);
    }
  }

  __global__ void __launch_bounds__(LST_LB_T3) kCreateT3(DeviceES es, const EventView* evs) {
    __shared__ T3Scratch sScratch[kT3Warps];
    const EventView& ev = evs[blockIdx.y];
    const int wib = threadIdx.x >> 5;
    // modules from the event's counter (kTaskCountersReset zeroes it before)
    for (unsigned int w = warpNextTask(&ev.sc->t3Next); w < es.nLowerModules; w = warpNextTask(&ev.sc->t3Next)) {
      __syncwarp();
      t3Module(es, ev, static_cast<uint16_t>(w), sScratch[wib]);
    }
  }

  // SDL/Triplet.h:1104-1122
  __global__ void kT3Ranges(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    for (unsigned int i = blockIdx.x * blockDim.x + threadIdx.x; i < es.nLowerModules; i += gridDim.x * blockDim.x) {
      if (ev.t3.nTriplets[i] == 0) {
        ev.rg.tripletRanges[i * 2] = -1;
        ev.rg.tripletRanges[i * 2 + 1] = -1;
      } else {
        ev.rg.tripletRanges[i * 2] = ev.rg.tripletModuleIndices[i];
        ev.rg.tripletRanges[i * 2 + 1] = ev.rg.tripletModuleIndices[i] + ev.t3.nTriplets[i] - 1;
      }
    }
  }

  // ========================================================= quintuplets
  // Eligible T5 seed modules and their offsets (SDL/Quintuplet.h:3117-3213).
  // Each thread takes a contiguous range of modules, so that one block scan
  // of the per-thread sums gives every eligible module its place.
  __global__ void __launch_bounds__(1024) kT5Eligible(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned int n = es.nLowerModules;
    const unsigned int per = (n + blockDim.x - 1) / blockDim.x;
    const unsigned int i0 = min(threadIdx.x * per, n), i1 = min(i0 + per, n);
    auto eligible = [&](unsigned int i) { return ev.t3.nTriplets[i] != 0 && es.t5CapIfEligible[i] >= 0; };
    unsigned int myN = 0, myQ = 0;
    for (unsigned int i = i0; i < i1; ++i)
      if (eligible(i)) {
        ++myN;
        myQ += static_cast<unsigned int>(es.t5CapIfEligible[i]);
      }
    unsigned int totN, totQ;
    unsigned int runN = blockExclusiveScan(myN, totN);
    unsigned int runQ = blockExclusiveScan(myQ, totQ);
    for (unsigned int i = i0; i < i1; ++i) {
      if (!eligible(i))
        continue;
      const unsigned int occ = static_cast<unsigned int>(es.t5CapIfEligible[i]);
      ev.rg.indicesOfEligibleT5Modules[runN++] = static_cast<uint16_t>(i);
      ev.rg.quintupletModuleIndices[i] = static_cast<int>(runQ);
      ev.rg.quintupletModuleOccupancy[i] = static_cast<int>(occ);
      runQ += occ;
    }
    if (threadIdx.x == 0) {
      *ev.rg.nEligibleT5Modules = static_cast<uint16_t>(totN);
      *ev.rg.device_nTotalQuints = totQ;
    }
  }

  // One warp per eligible module walking (inner T3, outer T3) in order
  // (SDL/Quintuplet.h:2988-3115).
  constexpr int kT5Warps = 4;
  constexpr int kT5MaxInner = 1024;
  __device__ __forceinline__ void t5Module(
      DeviceES const& es, const EventView& ev, uint16_t lm1, unsigned int* pre, bool useDnn) {
    const Modules& m = es.m;
    const int layer = m.layers[lm1];
    if (layer != 1 && layer != 2)
      return;
    const unsigned int nInner = ev.t3.nTriplets[lm1];
    const unsigned int t3Base = ev.rg.tripletModuleIndices[lm1];
    const Triplets& t3r = ev.t3;
    // Only outer triplets whose first MD is the inner triplet's third MD can
    // pass (the first test of the reference's quintuplet algorithm); they are
    // enumerated through the MD-keyed triplet index in storage order.
    const unsigned int total = warpPrefix(pre, int(nInner), [&](int i) {
      uint16_t lm3 = t3r.lowerModuleIndices[3 * (t3Base + i) + 2];
      if (t3r.nTriplets[lm3] == 0)
        return 0u;
      const unsigned int seg2 = t3r.segmentIndices[2 * (t3Base + i) + 1];
      return static_cast<unsigned int>(ev.mdT3Count[ev.ls.mdIndices[2 * seg2 + 1]]);
    });
    const int cap = ev.rg.quintupletModuleOccupancy[lm1];
    const unsigned int base = ev.rg.quintupletModuleIndices[lm1];
    Triplets t3 = ev.t3;
    Quintuplets t5 = ev.t5;
    ConstDnn dnn;
    unsigned int count = 0;
    for (unsigned int start = 0; start < total; start += 32) {
      unsigned int f = start + laneId();
      bool ok = false;
      T5Values v;
      unsigned int innerT3 = 0, outerT3 = 0;
      uint16_t lm[5] = {lm1, 0, 0, 0, 0};
      if (f < total) {
        int i = findSlot(pre, int(nInner), f);
        innerT3 = t3Base + i;
        lm[1] = t3.lowerModuleIndices[3 * innerT3 + 1];
        lm[2] = t3.lowerModuleIndices[3 * innerT3 + 2];
        const unsigned int mdMid = ev.ls.mdIndices[2 * t3.segmentIndices[2 * innerT3 + 1] + 1];
        const unsigned int outerBase = ev.rg.tripletModuleIndices[lm[2]];
        outerT3 = outerBase + ev.t3ByMD[outerBase + ev.mdT3Start[mdMid] + (f - pre[i])];
        lm[3] = t3.lowerModuleIndices[3 * outerT3 + 1];
        lm[4] = t3.lowerModuleIndices[3 * outerT3 + 2];
        ok = t5Select(m, ev.md, ev.ls, t3, dnn.get(), useDnn, c_t5dnnWP, lm, innerT3, outerT3, v);
      }
      unsigned int tot;
      unsigned int r = count + warpRank(ok, tot);
      if (ok && int(r) < cap)
        storeT5(ev.md, ev.ls, t3, t5, innerT3, outerT3, lm, layer, v, base + r);
      count += tot;
    }
    if (laneId() == 0) {
      t5.nQuintuplets[lm1] = (int(count) < cap) ? count : (cap > 0 ? unsigned(cap) : 0u);
      t5.totOccupancyQuintuplets[lm1] = count;
      if (int(count) > cap)
        atomicOr(&ev.sc->status, kStatusCapOverflow);
    }
  }

  // ------------------------------------------ T5 as a candidate work list
  // The warp-per-module walk above leaves most lanes idle: a few modules own
  // most candidates and the candidates diverge early.  The batched path
  // instead (1) stores each module's candidate prefix over its inner
  // triplets, (2) scans module totals, (3) evaluates every candidate on its
  // own thread, and (4) walks each module's pass flags in candidate order,
  // re-evaluating only the passing candidates to store them at their rank.
  // Candidate c of module w is the c-th (inner, outer) pair of the walk, so
  // ranks, caps and stored values are those of the walk.  Events with more
  // candidates than the flag buffer holds take the walk instead.
  constexpr unsigned int kT5CandCap = 1u << 21;  // candidates per event
  constexpr unsigned int kCandQueueCap = 1u << 18;  // pre-selected candidates per event (T5, pT5, pT3)
  constexpr unsigned int kPixChunkCap = 1u << 16;   // 32-candidate chunks of the pT5 / pT3 chunk table
  constexpr unsigned int kT5SortCap = 1u << 15;     // quintuplets per event sorted by eta for the TC cleaning
  constexpr unsigned int kT5PassCap = 1u << 16;  // passing candidates per event whose values are kept

  __device__ __forceinline__ unsigned int t5CandidatesOf(const EventView& ev, unsigned int innerT3) {
    const Triplets& t3 = ev.t3;
    uint16_t lm3 = t3.lowerModuleIndices[3 * innerT3 + 2];
    if (t3.nTriplets[lm3] == 0)
      return 0u;
    const unsigned int seg2 = t3.segmentIndices[2 * innerT3 + 1];
    return static_cast<unsigned int>(ev.mdT3Count[ev.ls.mdIndices[2 * seg2 + 1]]);
  }

  // (inner, outer) triplets of candidate f of module lm1.
  __device__ __forceinline__ void t5Candidate(const EventView& ev, unsigned int t3Base, unsigned int nInner, unsigned int f,
                                              unsigned int& innerT3, unsigned int& outerT3) {
    const unsigned int* pre = ev.t5CandPre + t3Base;
    int lo = 0, hi = int(nInner);
    while (hi - lo > 1) {
      int mid = (lo + hi) >> 1;
      if (pre[mid] <= f)
        lo = mid;
      else
        hi = mid;
    }
    innerT3 = t3Base + lo;
    const Triplets& t3 = ev.t3;
    const unsigned int mdMid = ev.ls.mdIndices[2 * t3.segmentIndices[2 * innerT3 + 1] + 1];
    const unsigned int outerBase = ev.rg.tripletModuleIndices[t3.lowerModuleIndices[3 * innerT3 + 2]];
    outerT3 = outerBase + ev.t3ByMD[outerBase + ev.mdT3Start[mdMid] + (f - pre[lo])];
  }

  __global__ void kT5Prefix(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    const int wpb = blockDim.x >> 5;
    const int nE = *ev.rg.nEligibleT5Modules;
    for (int w = blockIdx.x * wpb + (threadIdx.x >> 5); w < nE; w += gridDim.x * wpb) {
      const uint16_t lm1 = ev.rg.indicesOfEligibleT5Modules[w];
      const int layer = es.m.layers[lm1];
      unsigned int carry = 0;
      if (layer == 1 || layer == 2) {
        const unsigned int nInner = ev.t3.nTriplets[lm1];
        const unsigned int t3Base = ev.rg.tripletModuleIndices[lm1];
        for (unsigned int b = 0; b < nInner; b += 32) {
          unsigned int i = b + laneId();
          unsigned int c = i < nInner ? t5CandidatesOf(ev, t3Base + i) : 0u;
          unsigned int incl = c;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            unsigned int y = __shfl_up_sync(kFullMask, incl, o);
            if (int(laneId()) >= o)
              incl += y;
          }
          if (i < nInner)
            ev.t5CandPre[t3Base + i] = carry + incl - c;
          carry += __shfl_sync(kFullMask, incl, 31);
        }
      }
      if (laneId() == 0)
        ev.t5ModCand[w] = carry;
    }
  }

  __global__ void __launch_bounds__(1024) kT5ModScan(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned int nE = *ev.rg.nEligibleT5Modules;
    unsigned int carry = 0;
    for (unsigned int base = 0; base < nE; base += blockDim.x) {
      unsigned int i = base + threadIdx.x;
      unsigned int c = i < nE ? ev.t5ModCand[i] : 0u;
      unsigned int tot;
      unsigned int ex = blockExclusiveScan(c, tot);
      if (i < nE)
        ev.t5ModOff[i] = carry + ex;
      carry += tot;
    }
    if (threadIdx.x == 0) {
      ev.t5ModOff[nE] = carry;
      ev.sc->t5CandTotal = carry;
      ev.sc->t5CandOverflow = (carry > kT5CandCap || ev.forceWalk) ? 1u : 0u;
      ev.sc->t5PassCount = 0;
      ev.sc->t5QueueCount = 0;
      ev.sc->t5QueueBack = 0;
    }
    // The chunk table: candidate 32 j lies in eligible module t5ChunkMod[j]
    // (filled whenever the candidates are decoded, i.e. without overflow).
    if (carry > kT5CandCap)
      return;
    __syncthreads();
    for (unsigned int i = threadIdx.x; i < nE; i += blockDim.x) {
      const unsigned int a = ev.t5ModOff[i], b = ev.t5ModOff[i + 1];
      for (unsigned int j = (a + 31u) >> 5; j < ((b + 31u) >> 5); ++j)
        ev.t5ChunkMod[j] = i;
    }
  }

  // (inner T3, outer T3, lower modules) of quintuplet candidate c.
  __device__ __forceinline__ void t5Decode(const EventView& ev, unsigned int c, unsigned int& innerT3,
                                           unsigned int& outerT3, uint16_t* lm) {
    // The largest w with off[w] <= c: from the chunk table and a short walk
    // (eligible modules without candidates are stepped over).
    const unsigned int* off = ev.t5ModOff;
    int lo = static_cast<int>(ev.t5ChunkMod[c >> 5]);
    while (off[lo + 1] <= c)
      ++lo;
    const uint16_t lm1 = ev.rg.indicesOfEligibleT5Modules[lo];
    t5Candidate(ev, ev.rg.tripletModuleIndices[lm1], ev.t3.nTriplets[lm1], c - off[lo], innerT3, outerT3);
    lm[0] = lm1;
    lm[1] = ev.t3.lowerModuleIndices[3 * innerT3 + 1];
    lm[2] = ev.t3.lowerModuleIndices[3 * innerT3 + 2];
    lm[3] = ev.t3.lowerModuleIndices[3 * outerT3 + 1];
    lm[4] = ev.t3.lowerModuleIndices[3 * outerT3 + 2];
  }

  // Pre-selection of the quintuplet candidates: the shared-MD and radius tests
  // that open the selection, which most candidates fail.  A failing candidate
  // gets its flag here; the survivors are queued in any order for kT5Eval,
  // which then runs the long tests with all lanes of a warp busy (a
  // candidate's outcome does not depend on the thread that evaluates it).
  // Candidates on all-barrel module patterns fill the queue from the front,
  // the others from the back, so that a warp mostly runs one set of the
  // tracklet algorithms.  A full queue makes kT5Eval evaluate every candidate.
  __global__ void __launch_bounds__(256) kT5Pre(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    if (ev.sc->t5CandOverflow)
      return;
    const unsigned int total = ev.sc->t5CandTotal;
    const unsigned int stride = gridDim.x * blockDim.x;
    for (unsigned int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < total; base += stride) {
      const unsigned int c = base + laneId();
      bool pass = false, mixed = false;
      if (c < total) {
        unsigned int innerT3, outerT3;
        uint16_t lm[5];
        t5Decode(ev, c, innerT3, outerT3, lm);
        T5Values v;
        T5Stage st;
        pass = t5RadiusStage(es.m, ev.md, ev.ls, ev.t3, lm, innerT3, outerT3, v, st);
        if (!pass)
          ev.t5CandFlag[c] = 0;
        else
          mixed = st.kind > 0;
      }
      const unsigned int maskF = __ballot_sync(kFullMask, pass && !mixed);
      const unsigned int maskB = __ballot_sync(kFullMask, pass && mixed);
      if ((maskF | maskB) == 0u)
        continue;
      unsigned int startF = 0, startB = 0;
      if (laneId() == 0) {
        if (maskF)
          startF = atomicAdd(&ev.sc->t5QueueCount, __popc(maskF));
        if (maskB)
          startB = atomicAdd(&ev.sc->t5QueueBack, __popc(maskB));
      }
      startF = __shfl_sync(kFullMask, startF, 0);
      startB = __shfl_sync(kFullMask, startB, 0);
      if (pass) {
        const unsigned int k = mixed ? startB + __popc(maskB & lanesBelowMask())
                                     : startF + __popc(maskF & lanesBelowMask());
        if (k < kCandQueueCap)
          ev.candQueue[mixed ? kCandQueueCap - 1 - k : k] = c;
      }
    }
  }

  // Records a candidate that passes the T5 selection: its values go to the
  // pass buffer (flag = slot + 1), or, when the buffer is full, the flag asks
  // for re-evaluation at emission (flag = kT5PassCap + 1).
  __device__ __forceinline__ void t5Keep(const EventView& ev, unsigned int c, const T5Values& v) {
    const unsigned int slot = atomicAdd(&ev.sc->t5PassCount, 1u);
    if (slot < kT5PassCap) {
      ev.t5PassValues[slot] = v;
      ev.t5PassC[slot] = c;
      ev.t5CandFlag[c] = slot + 1;
    } else {
      ev.t5CandFlag[c] = kT5PassCap + 1;
    }
  }

  // The T5 selection of the queued candidates with the DNN classifier in the
  // same kernel (SDL/Quintuplet.h:2921-2941 evaluates it inline).  Each
  // thread runs every test before the classifier on its candidates; a
  // candidate that reaches the classifier leaves its 38 inputs and its
  // selection state in the block's slice of the event's staging area (its
  // own rows, in L2) instead of running the 38-32-32-1 forward pass there
  // and then, on a few lanes of its warp.  When the block has evaluated all
  // of its candidates, its threads classify the block's staged candidates,
  // one per thread with the weights in shared memory, so that the forward
  // passes run on full warps.  A candidate that finds its block's slice full
  // is classified at once by its own thread; the arithmetic is the same
  // either way.
  __global__ void __launch_bounds__(LST_LB_T5EVAL) kT5Eval(DeviceES es, const EventView* evs, bool useDnn) {
    __shared__ T5DnnWeights sW;
    __shared__ unsigned int sCount;
    const EventView& ev = evs[blockIdx.y];
    if (ev.sc->t5CandOverflow)
      return;
    if (useDnn) {
      const float* src = reinterpret_cast<const float*>(&c_t5dnn);
      float* dst = reinterpret_cast<float*>(&sW);
      for (int i = threadIdx.x; i < kT5DnnParams; i += blockDim.x)
        dst[i] = src[i];
    }
    if (threadIdx.x == 0)
      sCount = 0;
    __syncthreads();
    const float wp = c_t5dnnWP;
    const unsigned int slice = kT5DnnCap / gridDim.x;
    const unsigned int base = blockIdx.x * slice;
    const unsigned int total = ev.sc->t5CandTotal;
    const unsigned int front = ev.sc->t5QueueCount, back = ev.sc->t5QueueBack;
    const bool fromQueue = front <= kCandQueueCap && back <= kCandQueueCap - front;
    const unsigned int n = fromQueue ? front + back : total;
    for (unsigned int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
      const unsigned int c = fromQueue ? ev.candQueue[q < front ? q : kCandQueueCap - 1 - (q - front)] : q;
      unsigned int innerT3, outerT3;
      uint16_t lm[5];
      t5Decode(ev, c, innerT3, outerT3, lm);
      T5Values v;
      T5Stage st;
      if (!t5SelectPre(es.m, ev.md, ev.ls, ev.t3, lm, innerT3, outerT3, v, st)) {
        ev.t5CandFlag[c] = 0;
        continue;
      }
      const unsigned int k = useDnn ? atomicAdd(&sCount, 1u) : slice;
      if (k < slice) {
        float feat[38];
        t5DnnFeatures(es.m, ev.md, ev.ls, ev.t3, st.xs, st.ys, st.mdIdx, lm, innerT3, v.innerRadius, v.outerRadius,
                      v.bridgeRadius, feat);
        for (int i = 0; i < 38; ++i)
          ev.t5DnnFeat[size_t(base + k) * 38 + i] = feat[i];
        T5DnnSlotG& sl = ev.t5DnnSlot[base + k];
        sl.v = v;
        for (int i = 0; i < 5; ++i) {
          sl.mdIdx[i] = st.mdIdx[i];
          sl.lm[i] = lm[i];
        }
        sl.cand = c;
        sl.tight = st.tight ? 1 : 0;
      } else if (t5Classify(es.m, ev.md, ev.ls, ev.t3, sW, useDnn, wp, lm, innerT3, v, st)) {
        t5Keep(ev, c, v);
      } else {
        ev.t5CandFlag[c] = 0;
      }
    }
    __syncthreads();
    const unsigned int m = sCount < slice ? sCount : slice;
    for (unsigned int k = threadIdx.x; k < m; k += blockDim.x) {
      float feat[38];
      for (int i = 0; i < 38; ++i)
        feat[i] = ev.t5DnnFeat[size_t(base + k) * 38 + i];
      const float inference = t5DnnForward(sW, feat);
      const T5DnnSlotG& sl = ev.t5DnnSlot[base + k];
      if (!(inference > wp)) {
        ev.t5CandFlag[sl.cand] = 0;
        continue;
      }
      T5Values v = sl.v;
      t5NonAnchor(es.m, ev.md, sl.lm, sl.mdIdx, v);
      v.tightCutFlag = sl.tight != 0 and (inference > wp);
      t5Keep(ev, sl.cand, v);
    }
  }

  // The warp-per-module walk, for events whose candidates overflow the flag
  // buffer (a no-op for the others).
  // Register budget: this fallback does work only for events whose candidates
  // overflow the lists; for the others its blocks return at once, and the
  // budget lets more of them be resident, so the launch drains in fewer waves.
  __global__ void __launch_bounds__(128, 8) kT5Walk(DeviceES es, const EventView* evs, bool useDnn) {
    __shared__ unsigned int sPre[kT5Warps][kT5MaxInner + 1];
    const EventView& ev = evs[blockIdx.y];
    if (!ev.sc->t5CandOverflow)
      return;
    const int wib = threadIdx.x >> 5;
    const int nE = *ev.rg.nEligibleT5Modules;
    for (int w = blockIdx.x * kT5Warps + wib; w < nE; w += gridDim.x * kT5Warps) {
      __syncwarp();
      t5Module(es, ev, ev.rg.indicesOfEligibleT5Modules[w], sPre[wib], useDnn);
    }
  }

  // The passing quintuplet candidates stored in candidate order, one block per
  // event: their (candidate index, value slot) keys are bitonic-sorted in
  // shared memory, so that a candidate's position among the passing ones of
  // its module -- the reference's occupancy rank -- comes from two binary
  // searches.  Events with more passing candidates than kT5RankCap leave the
  // storing to kT5Emit's per-module walk.
  constexpr unsigned int kT5RankCap = 8192;
  constexpr size_t kT5RankSmem = kT5RankCap * sizeof(unsigned long long);
  __global__ void __launch_bounds__(1024) kT5RankEmit(DeviceES es, const EventView* evs) {
    extern __shared__ __align__(16) unsigned char rsm[];
    unsigned long long* sKey = reinterpret_cast<unsigned long long*>(rsm);
    const EventView& ev = evs[blockIdx.y];
    const unsigned int n = ev.sc->t5PassCount;
    if (ev.sc->t5CandOverflow || n > kT5RankCap || ev.forceWalk)
      return;
    unsigned int N = 1;
    while (N < n)
      N <<= 1;
    for (unsigned int t = threadIdx.x; t < N; t += blockDim.x)
      sKey[t] = t < n ? (static_cast<unsigned long long>(ev.t5PassC[t]) << 32) | t : ~0ull;
    __syncthreads();
    for (unsigned int k = 2; k <= N; k <<= 1) {
      for (unsigned int j = k >> 1; j > 0; j >>= 1) {
        for (unsigned int i = threadIdx.x; i < N; i += blockDim.x) {
          const unsigned int l = i ^ j;
          if (l > i) {
            const unsigned long long a = sKey[i], b = sKey[l];
            if (((i & k) == 0) == (a > b)) {
              sKey[i] = b;
              sKey[l] = a;
            }
          }
        }
        __syncthreads();
      }
    }
    const int nE = *ev.rg.nEligibleT5Modules;
    const unsigned int* off = ev.t5ModOff;
    // first sorted position whose candidate index is at least c
    auto lowerBound = [&](unsigned int c) {
      unsigned int lo = 0, hi = n;
      while (lo < hi) {
        const unsigned int mid = (lo + hi) >> 1;
        if (static_cast<unsigned int>(sKey[mid] >> 32) < c)
          lo = mid + 1;
        else
          hi = mid;
      }
      return lo;
    };
    Triplets t3 = ev.t3;
    Quintuplets t5 = ev.t5;
    for (unsigned int p = threadIdx.x; p < n; p += blockDim.x) {
      const unsigned int c = static_cast<unsigned int>(sKey[p] >> 32);
      const unsigned int slot = static_cast<unsigned int>(sKey[p] & 0xffffffffu);
      int lo = 0, hi = nE;  // module position w: largest with off[w] <= c
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (off[mid] <= c)
          lo = mid;
        else
          hi = mid;
      }
      const uint16_t lm1 = ev.rg.indicesOfEligibleT5Modules[lo];
      const int layer = es.m.layers[lm1];
      if (layer != 1 && layer != 2)
        continue;
      const unsigned int r = p - lowerBound(off[lo]);
      if (int(r) >= ev.rg.quintupletModuleOccupancy[lm1])
        continue;
      unsigned int innerT3, outerT3;
      t5Candidate(ev, ev.rg.tripletModuleIndices[lm1], t3.nTriplets[lm1], c - off[lo], innerT3, outerT3);
      uint16_t lm[5] = {lm1, t3.lowerModuleIndices[3 * innerT3 + 1], t3.lowerModuleIndices[3 * innerT3 + 2],
                        t3.lowerModuleIndices[3 * outerT3 + 1], t3.lowerModuleIndices[3 * outerT3 + 2]};
      storeT5(ev.md, ev.ls, t3, t5, innerT3, outerT3, lm, layer, ev.t5PassValues[slot],
              ev.rg.quintupletModuleIndices[lm1] + r);
    }
    for (int w = threadIdx.x; w < nE; w += blockDim.x) {
      const uint16_t lm1 = ev.rg.indicesOfEligibleT5Modules[w];
      const int layer = es.m.layers[lm1];
      if (layer != 1 && layer != 2)
        continue;
      const unsigned int count = lowerBound(off[w] + ev.t5ModCand[w]) - lowerBound(off[w]);
      const int cap = ev.rg.quintupletModuleOccupancy[lm1];
      t5.nQuintuplets[lm1] = (int(count) < cap) ? count : (cap > 0 ? unsigned(cap) : 0u);
      t5.totOccupancyQuintuplets[lm1] = count;
      if (int(count) > cap)
        atomicOr(&ev.sc->status, kStatusCapOverflow);
    }
  }

  // Register budget: this fallback does work only for events whose candidates
  // overflow the lists; for the others its blocks return at once, and the
  // budget lets more of them be resident, so the launch drains in fewer waves.
  __global__ void __launch_bounds__(256, 4) kT5Emit(DeviceES es, const EventView* evs, bool useDnn) {
    const EventView& ev = evs[blockIdx.y];
    if (ev.sc->t5CandOverflow || (ev.sc->t5PassCount <= kT5RankCap && !ev.forceWalk))
      return;
    const int wpb = blockDim.x >> 5;
    const int nE = *ev.rg.nEligibleT5Modules;
    ConstDnn dnn;
    for (int w = blockIdx.x * wpb + (threadIdx.x >> 5); w < nE; w += gridDim.x * wpb) {
      const uint16_t lm1 = ev.rg.indicesOfEligibleT5Modules[w];
      const int layer = es.m.layers[lm1];
      if (layer != 1 && layer != 2)
        continue;
      const unsigned int total = ev.t5ModCand[w];
      const unsigned int off = ev.t5ModOff[w];
      const unsigned int t3Base = ev.rg.tripletModuleIndices[lm1];
      const unsigned int nInner = ev.t3.nTriplets[lm1];
      const int cap = ev.rg.quintupletModuleOccupancy[lm1];
      const unsigned int base = ev.rg.quintupletModuleIndices[lm1];
      Triplets t3 = ev.t3;
      Quintuplets t5 = ev.t5;
      unsigned int count = 0;
      for (unsigned int start = 0; start < total; start += 32) {
        const unsigned int f = start + laneId();
        const unsigned int flag = f < total ? ev.t5CandFlag[off + f] : 0u;
        const bool ok = flag != 0;
        unsigned int tot;
        const unsigned int r = count + warpRank(ok, tot);
        if (ok && int(r) < cap) {
          unsigned int innerT3, outerT3;
          t5Candidate(ev, t3Base, nInner, f, innerT3, outerT3);
          uint16_t lm[5] = {lm1, t3.lowerModuleIndices[3 * innerT3 + 1], t3.lowerModuleIndices[3 * innerT3 + 2],
                            t3.lowerModuleIndices[3 * outerT3 + 1], t3.lowerModuleIndices[3 * outerT3 + 2]};
          T5Values v;
          if (flag <= kT5PassCap)
            v = ev.t5PassValues[flag - 1];
          else
            t5Select(es.m, ev.md, ev.ls, t3, dnn.get(), useDnn, c_t5dnnWP, lm, innerT3, outerT3, v);
          storeT5(ev.md, ev.ls, t3, t5, innerT3, outerT3, lm, layer, v, base + r);
        }
        count += tot;
      }
      if (laneId() == 0) {
        t5.nQuintuplets[lm1] = (int(count) < cap) ? count : (cap > 0 ? unsigned(cap) : 0u);
        t5.totOccupancyQuintuplets[lm1] = count;
        if (int(count) > cap)
          atomicOr(&ev.sc->status, kStatusCapOverflow);
      }
    }
  }

  // Classifier-stage probe: every T5 candidate that reaches the DNN decision,
  // with its features, the loaded weights' score, the cut-only decision and
  // its 10 hits, appended to the caller's buffers (order not fixed).
  struct T5ProbeOut {
    float* feat;      // capacity x 38
    float* score;     // capacity
    uint8_t* cutPass; // capacity
    uint8_t* rzTight; // capacity
    unsigned int* hits;  // capacity x 10 (event-local hit indices)
    int* eventIndex;     // capacity (slot)
    unsigned int capacity;
    unsigned int* count;
  };

  __global__ void kT5Probe(DeviceES es, const EventView* evs, int firstSlot, T5ProbeOut out) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned int total = ev.sc->t5CandTotal;
    const int nE = *ev.rg.nEligibleT5Modules;
    const unsigned int* off = ev.t5ModOff;
    ConstDnn dnn;
    for (unsigned int c = blockIdx.x * blockDim.x + threadIdx.x; c < total; c += gridDim.x * blockDim.x) {
      int lo = 0, hi = nE;
      while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (off[mid] <= c)
          lo = mid;
        else
          hi = mid;
      }
      const uint16_t lm1 = ev.rg.indicesOfEligibleT5Modules[lo];
      unsigned int innerT3, outerT3;
      t5Candidate(ev, ev.rg.tripletModuleIndices[lm1], ev.t3.nTriplets[lm1], c - off[lo], innerT3, outerT3);
      uint16_t lm[5] = {lm1,
                        ev.t3.lowerModuleIndices[3 * innerT3 + 1],
                        ev.t3.lowerModuleIndices[3 * innerT3 + 2],
                        ev.t3.lowerModuleIndices[3 * outerT3 + 1],
                        ev.t3.lowerModuleIndices[3 * outerT3 + 2]};
      T5Values v;
      T5Probe p;
      if (!t5Select(es.m, ev.md, ev.ls, ev.t3, dnn.get(), true, c_t5dnnWP, lm, innerT3, outerT3, v, &p))
        continue;
      const unsigned int slot = atomicAdd(out.count, 1u);
      if (slot >= out.capacity)
        continue;
      for (int k = 0; k < 38; ++k)
        out.feat[38 * size_t(slot) + k] = p.feat[k];
      out.score[slot] = p.dnnScore;
      out.cutPass[slot] = p.cutPass ? 1 : 0;
      out.rzTight[slot] = p.rzTight ? 1 : 0;
      for (int k = 0; k < 6; ++k)
        out.hits[10 * size_t(slot) + k] = ev.t3.hitIndices[6 * innerT3 + k];
      for (int k = 0; k < 4; ++k)
        out.hits[10 * size_t(slot) + 6 + k] = ev.t3.hitIndices[6 * outerT3 + 2 + k];
      out.eventIndex[slot] = firstSlot + int(blockIdx.y);
    }
  }

  // Number of hits two T5s share (SDL/Kernels.h:42-84).
  LST_DEV int sharedHitsT5(const Quintuplets& q, unsigned int ix, unsigned int jx) {
    int nMatched = 0;
    for (int i = 0; i < 10; i++) {
      unsigned int a = q.hitIndices[10 * ix + i];
      bool matched = false;
      for (int j = 0; j < 10; j++)
        if (a == q.hitIndices[10 * jx + j]) {
          matched = true;
          break;
        }
      if (matched)
        nMatched++;
    }
    return nMatched;
  }

  // Duplicate removal among the T5s of one module (SDL/Kernels.h:202-249).
  // Every pair (i < j) of a module is independent and only ever sets isDup
  // bit 1, so the pairs are spread over a block: a chunk of 32 entries of the
  // eligible-module list is scanned for modules holding two or more T5s, and each such module's
  // T5s are staged in shared memory (eta, phi, score, hits) and its n x n pair
  // square is shared out among the block's threads.  The largest modules hold
  // a few hundred T5s, whose pairs would otherwise run on one warp.
  constexpr int kT5DedupThreads = 128;
  constexpr unsigned int kT5DedupStage = 256;
  __global__ void __launch_bounds__(kT5DedupThreads) kT5DedupAfterBuild(DeviceES es, const EventView* evs) {
    __shared__ float sEta[kT5DedupStage], sPhi[kT5DedupStage], sScore[kT5DedupStage];
    __shared__ unsigned int sHits[kT5DedupStage * 10];
    __shared__ uint16_t sMods[32];
    __shared__ unsigned int sNMods;
    const EventView& ev = evs[blockIdx.y];
    const unsigned int nElig = *ev.rg.nEligibleT5Modules;
    Quintuplets q = ev.t5;
    // chunks of 32 eligible modules: the first warp picks those with two or more T5s
    for (unsigned int c0 = blockIdx.x * 32; c0 < nElig; c0 += gridDim.x * 32) {
      if (threadIdx.x < 32) {
        const unsigned int e = c0 + threadIdx.x;
        uint16_t lmLoad = 0;
        unsigned int nLoad = 0;
        if (e < nElig) {
          lmLoad = ev.rg.indicesOfEligibleT5Modules[e];
          nLoad = q.nQuintuplets[lmLoad];
        }
        unsigned int tot;
        const unsigned int slot = warpRank(nLoad >= 2, tot);
        if (nLoad >= 2)
          sMods[slot] = lmLoad;
        if (threadIdx.x == 0)
          sNMods = tot;
      }
      __syncthreads();
      const unsigned int nMods = sNMods;
      for (unsigned int k = 0; k < nMods; ++k) {
        const uint16_t lm = sMods[k];
        const unsigned int n = q.nQuintuplets[lm];
        const unsigned int base = ev.rg.quintupletModuleIndices[lm];
        const bool staged = n <= kT5DedupStage && !ev.forceWalk;
        if (staged) {
          for (unsigned int t = threadIdx.x; t < n; t += blockDim.x) {
            sEta[t] = q.eta[base + t];
            sPhi[t] = q.phi[base + t];
            sScore[t] = q.score_rphisum[base + t];
          }
          for (unsigned int t = threadIdx.x; t < 10 * n; t += blockDim.x)
            sHits[t] = q.hitIndices[10 * base + t];
        }
        __syncthreads();
        for (unsigned int pr = threadIdx.x; pr < n * n; pr += blockDim.x) {
          const unsigned int i = pr / n, j = pr - i * n;
          if (j <= i)
            continue;
          const unsigned int ix = base + i, jx = base + j;
          const float eta1 = staged ? sEta[i] : q.eta[ix], phi1 = staged ? sPhi[i] : q.phi[ix];
          const float eta2 = staged ? sEta[j] : q.eta[jx], phi2 = staged ? sPhi[j] : q.phi[jx];
          const float dEta = fabs_(eta1 - eta2);
          const float dPhi = wrapDPhi(phi1, phi2);
          if (dEta > 0.1f)
            continue;
          if (fabs_(dPhi) > 0.1f)
            continue;
          int nMatched = 0;
          if (staged) {
            for (int a = 0; a < 10; a++) {
              const unsigned int h = sHits[10 * i + a];
              bool matched = false;
              for (int b = 0; b < 10; b++)
                matched |= h == sHits[10 * j + b];
              nMatched += matched ? 1 : 0;
            }
          } else {
            nMatched = sharedHitsT5(q, ix, jx);
          }
          if (nMatched >= 7) {
            const float score1 = staged ? sScore[i] : q.score_rphisum[ix];
            const float score2 = staged ? sScore[j] : q.score_rphisum[jx];
            if (score1 >= score2)
              q.isDup[ix] = 1;
            else
              q.isDup[jx] = 1;
          }
        }
        __syncthreads();
      }
      __syncthreads();  // sMods / sNMods are rewritten for the next chunk
    }
  }

  // SDL/Quintuplet.h:3215-3235
  __global__ void kT5Ranges(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    for (unsigned int i = blockIdx.x * blockDim.x + threadIdx.x; i < es.nLowerModules; i += gridDim.x * blockDim.x) {
      if (ev.t5.nQuintuplets[i] == 0 or ev.rg.quintupletModuleIndices[i] == -1) {
        ev.rg.quintupletRanges[i * 2] = -1;
        ev.rg.quintupletRanges[i * 2 + 1] = -1;
      } else {
        ev.rg.quintupletRanges[i * 2] = ev.rg.quintupletModuleIndices[i];
        ev.rg.quintupletRanges[i * 2 + 1] = ev.rg.quintupletModuleIndices[i] + ev.t5.nQuintuplets[i] - 1;
      }
    }
  }

  // ==================================================== pLS cleaning
  // SDL/Kernels.h:384-473.  Pass 1 sets bit 1 of isDup directly; pass 2 marks
  // plsFlag and kMergePLSFlag folds it into bit 2 afterwards, so that pass 2
  // reads the pass-1 bit while other threads mark removals.
  // pLS binned by eta: bins of width 0.02 over [-6, 6) (clamped at both ends)
  // plus a last bin for non-finite eta, which must meet every pLS because a
  // NaN never satisfies the reference's |deta| > 0.1 skip.  Two etas within
  // 0.1 of each other land at most kPLSBinReach bins apart (5 bin widths plus
  // the rounding of the bin coordinate).
  constexpr int kPLSBins = 600;
  constexpr int kPLSBinReach = 6;
  LST_DEV int plsEtaBin(float eta) {
    if (!(fabsf(eta) <= 3.0e38f))
      return kPLSBins;
    float t = (eta + 6.0f) * 50.0f;
    if (t < 0.f)
      return 0;
    if (t >= float(kPLSBins))
      return kPLSBins - 1;
    return static_cast<int>(t);
  }

  // The removal of one tested pLS pair (SDL/Kernels.h:384-473): ix the lower
  // index (the reference's outer loop), jx the higher; marks the one to go.
  LST_DEV void plsRemoveOf(const EventView& ev, unsigned int ix, unsigned int jx, bool secondpass) {
    const Segments& s = ev.ls;
    const int8_t quad_diff = s.isQuad[ix] - s.isQuad[jx];
    const float score_diff = s.score[ix] - s.score[jx];
    unsigned int idxToRemove;
    if (quad_diff > 0)
      idxToRemove = jx;
    else if (quad_diff < 0)
      idxToRemove = ix;
    else if (score_diff < 0)
      idxToRemove = jx;
    else if (score_diff > 0)
      idxToRemove = ix;
    else
      idxToRemove = ix;
    if (secondpass)
      ev.plsFlag[idxToRemove] = 1;
    else
      s.isDup[idxToRemove] = 1;
  }

  LST_DEV bool plsCleanEligible(const Segments& s, unsigned int i, bool secondpass) {
    return !secondpass || (s.isQuad[i] && !(s.isDup[i] & 1));
  }

  // pLS duplicate removal (SDL/Kernels.h:384-473).  Pass 1 sets bit 1 of
  // isDup directly; pass 2 marks plsFlag and kMergePLSFlag folds it into bit 2
  // afterwards, so that pass 2 reads the pass-1 bit while other threads mark
  // removals.  The outcome of a pair (ix < jx) depends only on the two pLS, and
  // marks are only ever set, so any visiting order and any repeat visit give
  // the reference's result.  A pair removes a pLS
  //   pass 1: if ix has at least 3 of its 4 hits among jx's (npMatched >= 3),
  //   pass 2: if they have a hit in common (npMatched >= 1) or dR2 < 1e-5,
  // in both cases unless |deta| > 0.1 (a NaN never satisfies that skip), and
  // in pass 2 only between quads without a pass-1 mark.
  //
  // kPLSCleanHits finds every pair of the hit conditions: one thread per pLS
  // ix walks the hit index for its hits (pass 1: hits 0 and 1, one of which
  // is among jx's when three of the four are; pass 2: all four) and tests the
  // higher-index pLS jx found there.  A pair met through several hits is
  // tested again, which changes nothing.
  __global__ void kPLSCleanHits(DeviceES es, const EventView* evs, bool secondpass) {
    const EventView& ev = evs[blockIdx.y];
    const Segments& s = ev.ls;
    unsigned int nPix = s.nSegments[es.pixelModule];
    if (nPix > kMaxPixelSegments)
      nPix = kMaxPixelSegments;
    const unsigned int maxSteps = 4 * nPix;  // a chain holds each entry once: no walk takes more
    const uint4* hits = reinterpret_cast<const uint4*>(s.pLSHitsIdxs);
    for (unsigned int ix = blockIdx.x * blockDim.x + threadIdx.x; ix < nPix; ix += gridDim.x * blockDim.x) {
      if (!plsCleanEligible(s, ix, secondpass))
        continue;
      const uint4 h1 = hits[ix];
      const unsigned int h1a[4] = {h1.x, h1.y, h1.z, h1.w};
      const float eta1 = s.eta[ix];
      const int nSlots = secondpass ? 4 : 2;
      for (int slot = 0; slot < nSlots; ++slot) {
        const unsigned int h = h1a[slot];
        unsigned int steps = 0;
        for (unsigned int e = ev.plsHitHead[plsHitBucket(h)]; e != kPLSHitNone; e = ev.plsHitNext[e]) {
          if (++steps > maxSteps) {
            atomicOr(&ev.sc->status, kStatusInvalidInput);
            break;
          }
          const unsigned int jx = e >> 2;
          if (jx <= ix || jx >= nPix || s.pLSHitsIdxs[e] != h)
            continue;
          if (fabs_(s.eta[jx] - eta1) > 0.1f)
            continue;
          if (!plsCleanEligible(s, jx, secondpass))
            continue;
          bool remove = true;  // pass 2: a hit in common
          if (!secondpass) {
            const uint4 h2 = hits[jx];
            int npMatched = 0;
            for (int k = 0; k < 4; k++)
              if (h1a[k] == h2.x || h1a[k] == h2.y || h1a[k] == h2.z || h1a[k] == h2.w)
                npMatched++;
            remove = npMatched >= 3;
          }
          if (remove)
            plsRemoveOf(ev, ix, jx, secondpass);
        }
      }
    }
  }

  // One pass-2 pLS as kPLSCleanNear reads it, stored in eta-bin order so that
  // a tile of candidates is one coalesced read.
  struct __align__(16) PLSRec {
    float eta, phi;
    unsigned int index, pad;
  };

  // Counting sort, by eta bin, of the pLS that pass 2 tests (the quads
  // without a pass-1 mark), one block per event; writes the bin starts (the
  // last entry being the number of records) and the sorted records.
  __global__ void __launch_bounds__(1024) kPLSBin(DeviceES es, const EventView* evs) {
    __shared__ unsigned int sCount[kPLSBins + 1];
    __shared__ unsigned int sCursor[kPLSBins + 1];
    const EventView& ev = evs[blockIdx.y];
    const Segments& s = ev.ls;
    unsigned int nPix = s.nSegments[es.pixelModule];
    if (nPix > kMaxPixelSegments)
      nPix = kMaxPixelSegments;
    for (int b = threadIdx.x; b <= kPLSBins; b += blockDim.x)
      sCount[b] = 0;
    __syncthreads();
    for (unsigned int i = threadIdx.x; i < nPix; i += blockDim.x)
      if (plsCleanEligible(s, i, true))
        atomicAdd(&sCount[plsEtaBin(s.eta[i])], 1u);
    __syncthreads();
    unsigned int c = threadIdx.x <= kPLSBins ? sCount[threadIdx.x] : 0u;
    unsigned int tot;
    unsigned int ex = blockExclusiveScan(c, tot);
    if (threadIdx.x <= kPLSBins) {
      sCursor[threadIdx.x] = ex;
      ev.plsBinStart[threadIdx.x] = ex;
    }
    if (threadIdx.x == 0)
      ev.plsBinStart[kPLSBins + 1] = tot;
    __syncthreads();
    for (unsigned int i = threadIdx.x; i < nPix; i += blockDim.x) {
      if (!plsCleanEligible(s, i, true))
        continue;
      PLSRec r;
      r.eta = s.eta[i];
      r.phi = s.phi[i];
      r.index = i;
      r.pad = 0;
      ev.plsRec[atomicAdd(&sCursor[plsEtaBin(r.eta)], 1u)] = r;
    }
  }

  // kPLSCleanNear finds the pass-2 pairs of the dR2 condition.  dR2 < 1e-5
  // needs |deta| < 0.0032, so both lie in the same or adjacent eta bins, and
  // a NaN or infinite eta never passes (the non-finite bin is left out).  Each
  // pair is tested once, by the record that comes first in the eta-sorted
  // order: each block takes kPLSCleanTile consecutive finite records (one per
  // thread) and streams, through shared memory, the later records up to one
  // bin above its last record's bin; each warp tests only the part its own
  // records can reach.  dEta and dPhi are taken with the lower index first,
  // as in the reference.
  constexpr int kPLSCleanTile = 128;

  __global__ void __launch_bounds__(kPLSCleanTile) kPLSCleanNear(DeviceES es, const EventView* evs) {
    __shared__ PLSRec sT[kPLSCleanTile];
    const EventView& ev = evs[blockIdx.y];
    const PLSRec* rec = ev.plsRec;
    const unsigned int* binStart = ev.plsBinStart;
    const unsigned int nFinite = binStart[kPLSBins];
    const unsigned int warp = threadIdx.x >> 5;
    for (unsigned int k0 = blockIdx.x * kPLSCleanTile; k0 < nFinite; k0 += gridDim.x * kPLSCleanTile) {
      const unsigned int k = k0 + threadIdx.x;
      const bool active = k < nFinite;
      PLSRec me{};
      if (active)
        me = rec[k];
      const unsigned int kLast = min(k0 + kPLSCleanTile, nFinite) - 1;
      const unsigned int span = binStart[min(plsEtaBin(rec[kLast].eta) + 1, kPLSBins - 1) + 1] - k0;
      // this warp's part of the stream: offsets [tW0, tW1)
      const unsigned int kW0 = k0 + warp * 32;
      const unsigned int tW0 = warp * 32;
      unsigned int tW1 = 0;
      if (kW0 < nFinite) {
        const unsigned int kW1 = min(kW0 + 32, nFinite) - 1;
        tW1 = binStart[min(plsEtaBin(rec[kW1].eta) + 1, kPLSBins - 1) + 1] - k0;
      }
      for (unsigned int t0 = 0; t0 < span; t0 += kPLSCleanTile) {
        __syncthreads();
        const unsigned int t = t0 + threadIdx.x;
        if (t < span)
          sT[threadIdx.x] = rec[k0 + t];
        __syncthreads();
        if (!active)
          continue;
        const unsigned int nt = min(span - t0, unsigned(kPLSCleanTile));
        const unsigned int uEnd = tW1 > t0 ? min(tW1 - t0, nt) : 0u;
        for (unsigned int u = tW0 > t0 ? tW0 - t0 : 0u; u < uEnd; ++u) {
          if (t0 + u <= threadIdx.x)
            continue;
          const PLSRec o = sT[u];
          const bool meLow = me.index < o.index;
          const float eta1 = meLow ? me.eta : o.eta, eta2 = meLow ? o.eta : me.eta;
          const float phi1 = meLow ? me.phi : o.phi, phi2 = meLow ? o.phi : me.phi;
          const float dEta = fabs_(eta1 - eta2);
          const float dPhi = wrapDPhi(phi1, phi2);
          const float dR2 = dEta * dEta + dPhi * dPhi;
          if (dR2 < 1e-5f)
            plsRemoveOf(ev, meLow ? me.index : o.index, meLow ? o.index : me.index, true);
        }
      }
    }
  }

  __global__ void kMergePLSFlag(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    unsigned int nPix = ev.ls.nSegments[es.pixelModule];
    if (nPix > kMaxPixelSegments)
      nPix = kMaxPixelSegments;
    for (unsigned int i = blockIdx.x * blockDim.x + threadIdx.x; i < nPix; i += gridDim.x * blockDim.x) {
      if (ev.plsFlag[i]) {
        ev.ls.isDup[i] |= 2;
        ev.plsFlag[i] = 0;
      }
    }
  }

  // ============================================ pixel-map slices per pLS
  // SDL/Event.cc:1055-1080
  __global__ void kPixelConnect(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned int nPLS = ev.ls.nSegments[es.pixelModule];
    for (unsigned int i = blockIdx.x * blockDim.x + threadIdx.x; i < nPLS; i += gridDim.x * blockDim.x) {
      int8_t pixelType = ev.ls.pixelType[i];
      int superbin = ev.ls.superbin[i];
      unsigned int size = 0, index = 0;
      if (!((superbin < 0) or (superbin >= int(kSizeSuperbins)) or (pixelType > 2) or (pixelType < 0))) {
        if (pixelType == 0) {
          size = es.cpSizes[superbin];
          index = es.cpIndex[superbin];
        } else if (pixelType == 1) {
          size = es.cpSizesPos[superbin];
          index = es.cpIndexPos[superbin] + es.pixelIndexOffsetPos;
        } else {
          size = es.cpSizesNeg[superbin];
          index = es.cpIndexNeg[superbin] + es.pixelIndexOffsetNeg;
        }
      }
      ev.plsConnSize[i] = size;
      ev.plsConnIndex[i] = index;
    }
  }

  // ============================================================== pT5
  // Candidate modules of a pLS for pT5 (SDL/PixelTriplet.h:2697-2716).
  __device__ __forceinline__ unsigned int pt5ModuleCount(DeviceES const& es, const EventView& ev, uint16_t mod) {
    if (mod >= es.nLowerModules)
      return 0;
    if (es.m.moduleType[mod] == TwoS)
      return 0;
    return ev.t5.nQuintuplets[mod];
  }

  // Walks the pT5 candidates of one pLS in order; emit selects the pass:
  // count passing candidates, or store those with global rank < cap.
  constexpr int kPixWarps = 4;
  template <bool kEmit>
  __device__ __forceinline__ void pt5Walk(DeviceES const& es, const EventView& ev, unsigned int iPLS, unsigned int* pre,
                                          uint16_t* mods) {
    if (ev.ls.isDup[iPLS])
      return;
    const unsigned int nConn = ev.plsConnSize[iPLS];
    const unsigned int cidx = ev.plsConnIndex[iPLS];
    for (unsigned int k = laneId(); k < nConn; k += 32)
      mods[k] = static_cast<uint16_t>(es.m.connectedPixels[cidx + k]);
    __syncwarp();
    const unsigned int total = warpPrefix(pre, int(nConn), [&](int k) { return pt5ModuleCount(es, ev, mods[k]); });
    const unsigned int plsIndex = es.lsOffset[es.nLowerModules] + iPLS;
    unsigned int count = 0;
    unsigned int rankBase = kEmit ? ev.plsOffset[iPLS] : 0u;
    Segments ls = ev.ls;
    Triplets t3 = ev.t3;
    Quintuplets t5 = ev.t5;
    PixelQuintuplets pt5 = ev.pt5;
    for (unsigned int start = 0; start < total; start += 32) {
      unsigned int f = start + laneId();
      bool ok = false;
      PT5Values v;
      unsigned int t5i = 0;
      if (f < total) {
        int k = findSlot(pre, int(nConn), f);
        t5i = ev.rg.quintupletModuleIndices[mods[k]] + (f - pre[k]);
        if (!t5.isDup[t5i])
          ok = pt5Select(es.m, ev.rg, ev.md, ls, t3, t5, plsIndex, t5i, iPLS, v);
      }
      unsigned int tot;
      unsigned int r = rankBase + count + warpRank(ok, tot);
      if (kEmit && ok && r < kMaxPixelQuintuplets)
        storePT5(ev.md, ls, t3, t5, pt5, plsIndex, iPLS, t5i, v, r);
      count += tot;
    }
    if (!kEmit && laneId() == 0)
      ev.plsCount[iPLS] = count;
  }

  // Register budget: this fallback does work only for events whose candidates
  // overflow the lists; for the others its blocks return at once, and the
  // budget lets more of them be resident, so the launch drains in fewer waves.
  __global__ void __launch_bounds__(128, 8) kPT5Count(DeviceES es, const EventView* evs) {
    __shared__ unsigned int sPre[kPixWarps][kMaxConnectedModules + 1];
    __shared__ uint16_t sMods[kPixWarps][kMaxConnectedModules];
    const EventView& ev = evs[blockIdx.y];
    if (!ev.sc->pixFallback)
      return;
    const int wib = threadIdx.x >> 5;
    const unsigned int nPLS = ev.ls.nSegments[es.pixelModule];
    for (unsigned int i = blockIdx.x * kPixWarps + wib; i < nPLS; i += gridDim.x * kPixWarps) {
      __syncwarp();
      if (laneId() == 0)
        ev.plsCount[i] = 0;
      pt5Walk<false>(es, ev, i, sPre[wib], sMods[wib]);
    }
  }

  // Register budget: this fallback does work only for events whose candidates
  // overflow the lists; for the others its blocks return at once, and the
  // budget lets more of them be resident, so the launch drains in fewer waves.
  __global__ void __launch_bounds__(128, 8) kPT5Emit(DeviceES es, const EventView* evs) {
    __shared__ unsigned int sPre[kPixWarps][kMaxConnectedModules + 1];
    __shared__ uint16_t sMods[kPixWarps][kMaxConnectedModules];
    const EventView& ev = evs[blockIdx.y];
    if (!ev.sc->pixFallback)
      return;
    const int wib = threadIdx.x >> 5;
    const unsigned int nPLS = ev.ls.nSegments[es.pixelModule];
    for (unsigned int i = blockIdx.x * kPixWarps + wib; i < nPLS; i += gridDim.x * kPixWarps) {
      __syncwarp();
      if (ev.plsCount[i] == 0 || ev.plsOffset[i] >= kMaxPixelQuintuplets)
        continue;
      pt5Walk<true>(es, ev, i, sPre[wib], sMods[wib]);
    }
  }

  // Exclusive scan of the per-pLS pass counts; one block per event.
  // which = 0: pT5 (cap 15000), 1: pT3 (cap 5000).
  __global__ void __launch_bounds__(1024) kPLSScan(DeviceES es, const EventView* evs, int which) {
    const EventView& ev = evs[blockIdx.y];
    if (!ev.sc->pixFallback)
      return;
    const unsigned int n = ev.ls.nSegments[es.pixelModule];
    unsigned int carry = 0;
    for (unsigned int base = 0; base < n; base += blockDim.x) {
      unsigned int i = base + threadIdx.x;
      unsigned int c = (i < n) ? ev.plsCount[i] : 0u;
      unsigned int tot;
      unsigned int ex = blockExclusiveScan(c, tot);
      if (i < n)
        ev.plsOffset[i] = carry + ex;
      carry += tot;
    }
    if (threadIdx.x == 0) {
      if (which == 0) {
        ev.sc->nPT5Total = carry;
        *ev.pt5.totOccupancyPixelQuintuplets = carry;
        *ev.pt5.nPixelQuintuplets = carry < kMaxPixelQuintuplets ? carry : kMaxPixelQuintuplets;
      } else {
        ev.sc->nPT3Total = carry;
        *ev.pt3.totOccupancyPixelTriplets = carry;
        *ev.pt3.nPixelTriplets = carry < kMaxPixelTriplets ? carry : kMaxPixelTriplets;
      }
      if ((which == 0 && carry > kMaxPixelQuintuplets) || (which == 1 && carry > kMaxPixelTriplets))
        atomicOr(&ev.sc->status, kStatusCapOverflow);
    }
  }

  // pT5 duplicate removal (SDL/Kernels.h:356-382): pT5 ix is removed if some
  // jx shares at least 7 of its 14 hit slots and has a lower score (ties: the
  // higher index goes).  The outcome is an OR over jx, and a pair sharing 7
  // slots shares at least one hit, so only pairs that meet in some hit need the
  // full test.  kPT5DedupHashed (kPT5DedupBlocks blocks per event) chains the
  // event's (hit, pT5) entries by hit in a shared-memory hash table (a head
  // per bucket, a next index per entry, filled by one atomicExch per entry),
  // each block on its own, and tests its share of the entries against the
  // other entries of the same hit (the marks are only ever set, so the
  // blocks' marks combine and the walking order does not matter); an event
  // with more than kPT5DedupMaxN pT5s is left to kPT5Dedup, which tests every
  // pair in shared-memory tiles.
  constexpr unsigned int kPT5DedupBlocks = 2;
  constexpr unsigned int kPT5DedupMaxEntries = 16384;
  constexpr unsigned int kPT5DedupMaxN = kPT5DedupMaxEntries / 14;
  constexpr unsigned int kPT5DedupBucketBits = 13;
  constexpr unsigned int kPT5DedupBuckets = 1u << kPT5DedupBucketBits;
  constexpr unsigned int kPT5DedupNone = 0xffffffffu;
  constexpr size_t kPT5DedupSmem = kPT5DedupBuckets * sizeof(unsigned int) +
                                   2 * kPT5DedupMaxEntries * sizeof(unsigned int) +
                                   kPT5DedupMaxN * sizeof(float) + kPT5DedupMaxN;
  LST_DEV unsigned int pt5HitBucket(unsigned int h) { return (h * 2654435761u) >> (32 - kPT5DedupBucketBits); }

  __global__ void __launch_bounds__(1024) kPT5DedupHashed(DeviceES es, const EventView* evs) {
    extern __shared__ __align__(16) unsigned char psm[];
    unsigned int* sHead = reinterpret_cast<unsigned int*>(psm);
    unsigned int* sNext = sHead + kPT5DedupBuckets;
    unsigned int* sHits = sNext + kPT5DedupMaxEntries;
    float* sScore = reinterpret_cast<float*>(sHits + kPT5DedupMaxEntries);
    unsigned char* sDup = reinterpret_cast<unsigned char*>(sScore + kPT5DedupMaxN);
    const EventView& ev = evs[blockIdx.y];
    const unsigned int n = *ev.pt5.nPixelQuintuplets;
    if (n < 2 || n > kPT5DedupMaxN || ev.forceWalk)
      return;
    PixelQuintuplets p = ev.pt5;
    const unsigned int E = 14 * n;
    for (unsigned int t = threadIdx.x; t < kPT5DedupBuckets; t += blockDim.x)
      sHead[t] = kPT5DedupNone;
    for (unsigned int t = threadIdx.x; t < n; t += blockDim.x) {
      sScore[t] = p.score[t];
      sDup[t] = 0;
    }
    __syncthreads();
    for (unsigned int t = threadIdx.x; t < E; t += blockDim.x) {
      const unsigned int h = p.hitIndices[t];
      sHits[t] = h;
      sNext[t] = atomicExch(&sHead[pt5HitBucket(h)], t);
    }
    __syncthreads();
    for (unsigned int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
      const unsigned int a = e / 14;
      const unsigned int h = sHits[e];
      const float score1 = sScore[a];
      for (unsigned int q = sHead[pt5HitBucket(h)]; q != kPT5DedupNone; q = sNext[q]) {
        if (sDup[a])
          break;
        if (sHits[q] != h)
          continue;
        const unsigned int b = q / 14;
        if (b == a)
          continue;
        const float score2 = sScore[b];
        if (!(score1 > score2 or ((score1 == score2) and (a > b))))
          continue;
        const unsigned int* mine = sHits + 14 * a;
        const unsigned int* other = sHits + 14 * b;
        int nMatched = 0;
        for (int i = 0; i < 14; ++i) {
          bool matched = false;
          for (int j = 0; j < 14; ++j)
            matched |= (mine[i] == other[j]);
          nMatched += matched ? 1 : 0;
        }
        if (nMatched >= 7)
          sDup[a] = 1;
      }
    }
    __syncthreads();
    for (unsigned int t = threadIdx.x; t < n; t += blockDim.x)
      if (sDup[t])
        p.isDup[t] = 1;
  }

  constexpr int kDedupTile = 128;
  __global__ void __launch_bounds__(kDedupTile) kPT5Dedup(DeviceES es, const EventView* evs) {
    __shared__ unsigned int sHits[kDedupTile * 14];
    __shared__ float sScore[kDedupTile];
    const EventView& ev = evs[blockIdx.y];
    const unsigned int n = *ev.pt5.nPixelQuintuplets;
    if (n <= kPT5DedupMaxN && !ev.forceWalk)
      return;  // kPT5DedupHashed has done this event
    PixelQuintuplets p = ev.pt5;
    for (unsigned int ixBase = blockIdx.x * kDedupTile; ixBase < n; ixBase += gridDim.x * kDedupTile) {
      const unsigned int ix = ixBase + threadIdx.x;
      const bool valid = ix < n;
      unsigned int mine[14];
      float score1 = 0.f;
      if (valid) {
#pragma unroll
        for (int i = 0; i < 14; ++i)
          mine[i] = p.hitIndices[14 * ix + i];
        score1 = p.score[ix];
      }
      bool dup = false;
      for (unsigned int jBase = 0; jBase < n; jBase += kDedupTile) {
        const unsigned int tile = (n - jBase < kDedupTile) ? n - jBase : kDedupTile;
        __syncthreads();
        for (unsigned int t = threadIdx.x; t < tile * 14; t += blockDim.x)
          sHits[t] = p.hitIndices[14 * jBase + t];
        for (unsigned int t = threadIdx.x; t < tile; t += blockDim.x)
          sScore[t] = p.score[jBase + t];
        __syncthreads();
        if (!valid || dup)
          continue;
        for (unsigned int jj = 0; jj < tile; ++jj) {
          const unsigned int jx = jBase + jj;
          if (jx == ix)
            continue;
          const unsigned int* other = sHits + 14 * jj;
          int nMatched = 0;
#pragma unroll
          for (int i = 0; i < 14; ++i) {
            bool matched = false;
#pragma unroll
            for (int j = 0; j < 14; ++j)
              matched |= (mine[i] == other[j]);
            nMatched += matched ? 1 : 0;
          }
          const float score2 = sScore[jj];
          if (nMatched >= 7) {
            if (score1 > score2 or ((score1 == score2) and (ix > jx))) {
              dup = true;
              break;
            }
          }
        }
      }
      if (valid && dup)
        p.isDup[ix] = 1;
    }
  }

  // Writes a track candidate built from a pT3 / T5 / pT5 record
  // (SDL/TrackCandidate.h:130-163); unused slots are zeroed.
  LST_DEV void storeTC(TrackCandidates& tc,
                       short type,
                       unsigned int innerIdx,
                       unsigned int outerIdx,
                       const uint8_t* logicalLayers,
                       const uint16_t* lowerModules,
                       const unsigned int* hitIndices,
                       int pixelSeedIndex,
                       float centerX,
                       float centerY,
                       float radius,
                       unsigned int idx,
                       unsigned int directIdx) {
    tc.trackCandidateType[idx] = type;
    tc.directObjectIndices[idx] = directIdx;
    tc.pixelSeedIndex[idx] = pixelSeedIndex;
    tc.objectIndices[2 * idx] = innerIdx;
    tc.objectIndices[2 * idx + 1] = outerIdx;
    const int limits = type == 7 ? 7 : 5;
    for (int i = 0; i < 7; i++) {
      tc.logicalLayers[7 * idx + i] = i < limits ? logicalLayers[i] : 0;
      tc.lowerModuleIndices[7 * idx + i] = i < limits ? lowerModules[i] : 0;
    }
    for (int i = 0; i < 14; i++)
      tc.hitIndices[14 * idx + i] = i < 2 * limits ? hitIndices[i] : 0;
    tc.centerX[idx] = centerX;
    tc.centerY[idx] = centerY;
    tc.radius[idx] = radius;
  }

  // pT5 -> TC (SDL/TrackCandidate.h:531-581); one block per event.
  __global__ void __launch_bounds__(1024) kAddPT5TC(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned int n = *ev.pt5.nPixelQuintuplets;
    const unsigned int pLS_offset = es.lsOffset[es.nLowerModules];
    const unsigned int start = *ev.tc.nTrackCandidates;
    TrackCandidates tc = ev.tc;
    PixelQuintuplets p = ev.pt5;
    unsigned int carry = 0;
    for (unsigned int base = 0; base < n; base += blockDim.x) {
      unsigned int i = base + threadIdx.x;
      bool f = i < n && !p.isDup[i];
      unsigned int tot;
      unsigned int ex = blockExclusiveScan(f ? 1u : 0u, tot);
      unsigned int idx = start + carry + ex;
      if (f && idx < kMaxPixelTrackCandidates) {
        float radius = 0.5f * (p.pixelRadius[i] + p.quintupletRadius[i]);
        unsigned int pix = p.pixelIndices[i];
        storeTC(tc, 7, pix, p.T5Indices[i], &p.logicalLayers[7 * i], &p.lowerModuleIndices[7 * i], &p.hitIndices[14 * i],
                static_cast<int>(ev.ls.seedIdx[pix - pLS_offset]), p.centerX[i], p.centerY[i], radius, idx, i);
      }
      carry += tot;
    }
    if (threadIdx.x == 0) {
      unsigned int accepted = (start + carry <= kMaxPixelTrackCandidates) ? carry
                              : (start < kMaxPixelTrackCandidates ? kMaxPixelTrackCandidates - start : 0u);
      if (accepted < carry)
        atomicOr(&ev.sc->status, kStatusTCTruncated);
      *tc.nTrackCandidates = start + accepted;
      *tc.nTrackCandidatespT5 += accepted;
    }
  }

  // ============================================================== pT3
  // Candidate modules of a pLS for pT3 (SDL/PixelTriplet.h:1046-1081).
  __device__ __forceinline__ unsigned int pt3ModuleCount(DeviceES const& es, const EventView& ev, uint16_t mod) {
    if (mod >= es.nLowerModules)
      return 0;
    if (es.m.moduleType[mod] == TwoS)
      return 0;
    int layer = es.m.layers[mod];
    if (layer != 1 && layer != 2)
      return 0;
    return ev.t3.nTriplets[mod];
  }

  template <bool kEmit>
  __device__ __forceinline__ void pt3Walk(DeviceES const& es, const EventView& ev, unsigned int iPLS, unsigned int* pre,
                                          uint16_t* mods) {
    if (ev.ls.isDup[iPLS] || ev.ls.partOfPT5[iPLS])
      return;
    const unsigned int nConn = ev.plsConnSize[iPLS];
    const unsigned int cidx = ev.plsConnIndex[iPLS];
    for (unsigned int k = laneId(); k < nConn; k += 32)
      mods[k] = static_cast<uint16_t>(es.m.connectedPixels[cidx + k]);
    __syncwarp();
    const unsigned int total = warpPrefix(pre, int(nConn), [&](int k) { return pt3ModuleCount(es, ev, mods[k]); });
    const unsigned int plsIndex = es.lsOffset[es.nLowerModules] + iPLS;
    unsigned int count = 0;
    unsigned int rankBase = kEmit ? ev.plsOffset[iPLS] : 0u;
    Triplets t3 = ev.t3;
    PixelTriplets pt3 = ev.pt3;
    for (unsigned int start = 0; start < total; start += 32) {
      unsigned int f = start + laneId();
      bool ok = false;
      PT3Values v;
      unsigned int t3i = 0;
      short adj = 0;
      if (f < total) {
        int k = findSlot(pre, int(nConn), f);
        uint16_t mod = mods[k];
        adj = es.m.layers[mod] == 1 ? 1 : 0;
        t3i = ev.rg.tripletModuleIndices[mod] + (f - pre[k]);
        if (es.m.moduleType[t3.lowerModuleIndices[3 * t3i + 1]] != TwoS && !t3.partOfPT5[t3i])
          ok = pt3Select(es.m, ev.rg, ev.md, ev.ls, t3, plsIndex, t3i, true, v);
      }
      unsigned int tot;
      unsigned int r = rankBase + count + warpRank(ok, tot);
      if (kEmit && ok && r < kMaxPixelTriplets) {
        storePT3(es.m, ev.md, ev.ls, t3, pt3, plsIndex, iPLS, t3i, adj, v, r);
        t3.partOfPT3[t3i] = 1;
      }
      count += tot;
    }
    if (!kEmit && laneId() == 0)
      ev.plsCount[iPLS] = count;
  }

  // Register budget: this fallback does work only for events whose candidates
  // overflow the lists; for the others its blocks return at once, and the
  // budget lets more of them be resident, so the launch drains in fewer waves.
  __global__ void __launch_bounds__(128, 8) kPT3Count(DeviceES es, const EventView* evs) {
    __shared__ unsigned int sPre[kPixWarps][kMaxConnectedModules + 1];
    __shared__ uint16_t sMods[kPixWarps][kMaxConnectedModules];
    const EventView& ev = evs[blockIdx.y];
    if (!ev.sc->pixFallback)
      return;
    const int wib = threadIdx.x >> 5;
    const unsigned int nPLS = ev.ls.nSegments[es.pixelModule];
    for (unsigned int i = blockIdx.x * kPixWarps + wib; i < nPLS; i += gridDim.x * kPixWarps) {
      __syncwarp();
      if (laneId() == 0)
        ev.plsCount[i] = 0;
      pt3Walk<false>(es, ev, i, sPre[wib], sMods[wib]);
    }
  }

  // Register budget: this fallback does work only for events whose candidates
  // overflow the lists; for the others its blocks return at once, and the
  // budget lets more of them be resident, so the launch drains in fewer waves.
  __global__ void __launch_bounds__(128, 8) kPT3Emit(DeviceES es, const EventView* evs) {
    __shared__ unsigned int sPre[kPixWarps][kMaxConnectedModules + 1];
    __shared__ uint16_t sMods[kPixWarps][kMaxConnectedModules];
    const EventView& ev = evs[blockIdx.y];
    if (!ev.sc->pixFallback)
      return;
    const int wib = threadIdx.x >> 5;
    const unsigned int nPLS = ev.ls.nSegments[es.pixelModule];
    for (unsigned int i = blockIdx.x * kPixWarps + wib; i < nPLS; i += gridDim.x * kPixWarps) {
      __syncwarp();
      if (ev.plsCount[i] == 0 || ev.plsOffset[i] >= kMaxPixelTriplets)
        continue;
      pt3Walk<true>(es, ev, i, sPre[wib], sMods[wib]);
    }
  }

  // ------------------------------------- pT5 / pT3 as candidate lists
  // Candidate c of the event is the c-th (pLS, connected module, object) of
  // the reference's loop nest (SDL/PixelTriplet.h:1043-1158, :2697-2786), so
  // the global rank of a passing candidate is the number of passing
  // candidates with a smaller c.  Every candidate is evaluated on its own
  // thread; the passing ones are appended with their values and one block
  // per event ranks them by c and stores the first 15000 (pT5) / 5000 (pT3).
  // Events with more passing candidates than the staging holds take the
  // per-pLS count/emit walk instead.
  constexpr unsigned int kPixPassCap = 8192;
  constexpr int kConnStride = kMaxConnectedModules + 1;

  template <int K>
  __device__ __forceinline__ unsigned int pixModuleCount(DeviceES const& es, const EventView& ev, uint16_t mod) {
    return K == 5 ? pt5ModuleCount(es, ev, mod) : pt3ModuleCount(es, ev, mod);
  }

  template <int K>
  __device__ __forceinline__ bool pixSkipPLS(const EventView& ev, unsigned int i) {
    return K == 5 ? (ev.ls.isDup[i] != 0) : (ev.ls.isDup[i] || ev.ls.partOfPT5[i]);
  }

  template <int K>
  __global__ void kPixPrefix(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    const int wpb = blockDim.x >> 5;
    const unsigned int nPLS = ev.ls.nSegments[es.pixelModule];
    for (unsigned int i = blockIdx.x * wpb + (threadIdx.x >> 5); i < nPLS; i += gridDim.x * wpb) {
      unsigned int carry = 0;
      unsigned int* pre = ev.plsModPre + size_t(i) * kConnStride;
      if (!pixSkipPLS<K>(ev, i)) {
        const unsigned int nConn = ev.plsConnSize[i];
        const unsigned int cidx = ev.plsConnIndex[i];
        for (unsigned int b = 0; b < nConn; b += 32) {
          const unsigned int k = b + laneId();
          const unsigned int c =
              k < nConn ? pixModuleCount<K>(es, ev, static_cast<uint16_t>(es.m.connectedPixels[cidx + k])) : 0u;
          unsigned int incl = c;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            unsigned int y = __shfl_up_sync(kFullMask, incl, o);
            if (int(laneId()) >= o)
              incl += y;
          }
          if (k < nConn)
            pre[k] = carry + incl - c;
          carry += __shfl_sync(kFullMask, incl, 31);
        }
      }
      if (laneId() == 0)
        ev.plsCand[i] = carry;
    }
  }

  __global__ void __launch_bounds__(1024) kPixScan(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned int n = ev.ls.nSegments[es.pixelModule];
    unsigned int carry = 0;
    for (unsigned int base = 0; base < n; base += blockDim.x) {
      unsigned int i = base + threadIdx.x;
      unsigned int c = i < n ? ev.plsCand[i] : 0u;
      unsigned int tot;
      unsigned int ex = blockExclusiveScan(c, tot);
      if (i < n)
        ev.plsCandOff[i] = carry + ex;
      carry += tot;
    }
    if (threadIdx.x == 0) {
      ev.plsCandOff[n] = carry;
      ev.sc->pixCandTotal = carry;
      ev.sc->pixPassCount = 0;
      ev.sc->pixQueueCount = 0;
      ev.sc->pixQueueBack = 0;
      ev.sc->pixQueue2Count = 0;
    }
    // The chunk table: candidate 32 j lies in pLS pixChunkPLS[j].
    if (carry > 32u * kPixChunkCap)
      return;
    __syncthreads();
    for (unsigned int i = threadIdx.x; i < n; i += blockDim.x) {
      const unsigned int a = ev.plsCandOff[i], b = ev.plsCandOff[i + 1];
      for (unsigned int j = (a + 31u) >> 5; j < ((b + 31u) >> 5); ++j)
        ev.pixChunkPLS[j] = i;
    }
  }

  // (pLS, object) of candidate c.
  template <int K>
  __device__ __forceinline__ void pixCandidate(DeviceES const& es, const EventView& ev, unsigned int c, unsigned int& iPLS,
                                               unsigned int& obj, uint16_t& mod) {
    const unsigned int nPLS = ev.ls.nSegments[es.pixelModule];
    const unsigned int* off = ev.plsCandOff;
    // The last pLS whose first candidate is at most c: from the chunk table
    // and a short walk (pLS without candidates are stepped over), or by a
    // binary search when the candidates outnumber the table.
    int lo = 0;
    if (ev.sc->pixCandTotal <= 32u * kPixChunkCap) {
      lo = static_cast<int>(ev.pixChunkPLS[c >> 5]);
      while (off[lo + 1] <= c)
        ++lo;
    } else {
      int hi = int(nPLS);
      while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (off[mid] <= c)
          lo = mid;
        else
          hi = mid;
      }
    }
    iPLS = lo;
    const unsigned int f = c - off[lo];
    const unsigned int* pre = ev.plsModPre + size_t(lo) * kConnStride;
    int klo = 0, khi = int(ev.plsConnSize[lo]);
    while (khi - klo > 1) {
      int mid = (klo + khi) >> 1;
      if (pre[mid] <= f)
        klo = mid;
      else
        khi = mid;
    }
    mod = static_cast<uint16_t>(es.m.connectedPixels[ev.plsConnIndex[lo] + klo]);
    obj = (K == 5 ? static_cast<unsigned int>(ev.rg.quintupletModuleIndices[mod])
                  : static_cast<unsigned int>(ev.rg.tripletModuleIndices[mod])) +
          (f - pre[klo]);
  }

  // Pre-selection of the pT5 / pT3 candidates: the tests that come first in
  // kPixEval (object not removed or used, the pLS-triplet radius criterion),
  // which most candidates fail.  The survivors are queued in any order, so
  // that kPixEval runs its long selection with all lanes of a warp busy; the
  // outcome of a candidate does not depend on which thread evaluates it, and
  // the passing ones are ranked by candidate index afterwards.  Candidates
  // whose first pixel tracklet takes the barrel algorithm fill the queue from
  // the front, the endcap ones from the back, so that a warp mostly runs one
  // of the two.  A full queue makes kPixEval evaluate every candidate instead.
  template <int K>
  __global__ void __launch_bounds__(256) kPixPre(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned int total = ev.sc->pixCandTotal;
    const unsigned int plsBase = es.lsOffset[es.nLowerModules];
    const unsigned int stride = gridDim.x * blockDim.x;
    for (unsigned int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < total; base += stride) {
      const unsigned int c = base + laneId();
      bool pass = false, endcap = false;
      if (c < total) {
        unsigned int iPLS, obj;
        uint16_t mod;
        pixCandidate<K>(es, ev, c, iPLS, obj, mod);
        const unsigned int t3 = K == 5 ? ev.t5.tripletIndices[2 * obj] : obj;
        if (K == 5)
          pass = !ev.t5.isDup[obj] && pt3RadiusPass(es.m, ev.rg, ev.ls, ev.t3, plsBase + iPLS, t3);
        else
          pass = es.m.moduleType[ev.t3.lowerModuleIndices[3 * obj + 1]] != TwoS && !ev.t3.partOfPT5[obj] &&
                 pt3RadiusPass(es.m, ev.rg, ev.ls, ev.t3, plsBase + iPLS, obj);
        endcap = es.m.subdets[ev.t3.lowerModuleIndices[3 * t3]] == Endcap;
      }
      const unsigned int maskF = __ballot_sync(kFullMask, pass && !endcap);
      const unsigned int maskB = __ballot_sync(kFullMask, pass && endcap);
      if ((maskF | maskB) == 0u)
        continue;
      unsigned int startF = 0, startB = 0;
      if (laneId() == 0) {
        if (maskF)
          startF = atomicAdd(&ev.sc->pixQueueCount, __popc(maskF));
        if (maskB)
          startB = atomicAdd(&ev.sc->pixQueueBack, __popc(maskB));
      }
      startF = __shfl_sync(kFullMask, startF, 0);
      startB = __shfl_sync(kFullMask, startB, 0);
      if (pass) {
        const unsigned int k = endcap ? startB + __popc(maskB & lanesBelowMask())
                                      : startF + __popc(maskF & lanesBelowMask());
        if (k < kCandQueueCap)
          ev.candQueue[endcap ? kCandQueueCap - 1 - k : k] = c;
      }
    }
  }

  // Second pre-selection stage: the first pixel tracklet algorithm (of the
  // pLS with the triplet's, or the quintuplet's inner triplet's, inner
  // segment), the long test that few queued candidates pass.  Its survivors
  // are queued again, between the two ends of the first queue; without room
  // there, kPixEval takes the first queue instead.
  template <int K>
  __global__ void __launch_bounds__(LST_LB_PIXMID) kPixMid(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned int front = ev.sc->pixQueueCount, back = ev.sc->pixQueueBack;
    if (!(front <= kCandQueueCap && back <= kCandQueueCap - front))
      return;
    const unsigned int n = front + back, room = kCandQueueCap - n;
    const unsigned int plsBase = es.lsOffset[es.nLowerModules];
    const unsigned int stride = gridDim.x * blockDim.x;
    for (unsigned int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
      const unsigned int q = base + laneId();
      bool pass = false;
      unsigned int c = 0;
      if (q < n) {
        c = ev.candQueue[q < front ? q : kCandQueueCap - 1 - (q - front)];
        unsigned int iPLS, obj;
        uint16_t mod;
        pixCandidate<K>(es, ev, c, iPLS, obj, mod);
        const unsigned int t3 = K == 5 ? ev.t5.tripletIndices[2 * obj] : obj;
        pass = pt3FirstTracklet(es.m, ev.rg, ev.md, ev.ls, ev.t3, plsBase + iPLS, t3);
      }
      const unsigned int mask = __ballot_sync(kFullMask, pass);
      if (mask == 0u)
        continue;
      unsigned int start = 0;
      if (laneId() == 0)
        start = atomicAdd(&ev.sc->pixQueue2Count, __popc(mask));
      start = __shfl_sync(kFullMask, start, 0);
      const unsigned int k = start + __popc(mask & lanesBelowMask());
      if (pass && k < room)
        ev.candQueue[front + k] = c;
    }
  }

  template <int K>
  __global__ void __launch_bounds__(LST_LB_EVAL) kPixEval(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned int total = ev.sc->pixCandTotal;
    const unsigned int front = ev.sc->pixQueueCount, back = ev.sc->pixQueueBack;
    const bool fromQueue = front <= kCandQueueCap && back <= kCandQueueCap - front;
    const unsigned int n2 = ev.sc->pixQueue2Count;
    const bool fromQueue2 = fromQueue && n2 <= kCandQueueCap - front - back;
    const unsigned int n = fromQueue2 ? n2 : (fromQueue ? front + back : total);
    const unsigned int plsBase = es.lsOffset[es.nLowerModules];
    for (unsigned int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
      const unsigned int c = fromQueue2  ? ev.candQueue[front + q]
                             : fromQueue ? ev.candQueue[q < front ? q : kCandQueueCap - 1 - (q - front)]
                                         : q;
      unsigned int iPLS, obj;
      uint16_t mod;
      pixCandidate<K>(es, ev, c, iPLS, obj, mod);
      float vals[8];
      bool ok;
      if (K == 5) {
        PT5Values v;
        ok = !ev.t5.isDup[obj] && pt5Select(es.m, ev.rg, ev.md, ev.ls, ev.t3, ev.t5, plsBase + iPLS, obj, iPLS, v);
        vals[0] = v.rzChiSquared;
        vals[1] = v.rPhiChiSquared;
        vals[2] = v.rPhiChiSquaredInwards;
        vals[3] = v.pixelRadius;
        vals[4] = v.quintupletRadius;
        vals[5] = v.centerX;
        vals[6] = v.centerY;
        vals[7] = 0.f;
      } else {
        PT3Values v;
        ok = es.m.moduleType[ev.t3.lowerModuleIndices[3 * obj + 1]] != TwoS && !ev.t3.partOfPT5[obj] &&
             pt3Select(es.m, ev.rg, ev.md, ev.ls, ev.t3, plsBase + iPLS, obj, true, v);
        vals[0] = v.pixelRadius;
        vals[1] = v.pixelRadiusError;
        vals[2] = v.tripletRadius;
        vals[3] = v.centerX;
        vals[4] = v.centerY;
        vals[5] = v.rzChiSquared;
        vals[6] = v.rPhiChiSquared;
        vals[7] = v.rPhiChiSquaredInwards;
      }
      if (ok) {
        const unsigned int slot = atomicAdd(&ev.sc->pixPassCount, 1u);
        if (slot < kPixPassCap) {
          ev.pixPassC[slot] = c;
          ev.pixPassObj[slot] = obj;
          ev.pixPassPLS[slot] = iPLS;
#pragma unroll
          for (int k = 0; k < 8; ++k)
            ev.pixPassV[8 * slot + k] = vals[k];
        }
      }
    }
  }

  // Ranks the passing candidates by c and stores them; one block per event.
  template <int K>
  __global__ void __launch_bounds__(1024) kPixRankEmit(DeviceES es, const EventView* evs) {
    __shared__ unsigned int sKey[kPixPassCap];
    const EventView& ev = evs[blockIdx.y];
    const unsigned int n = ev.sc->pixPassCount;
    const unsigned int capOut = K == 5 ? kMaxPixelQuintuplets : kMaxPixelTriplets;
    if (n > kPixPassCap || ev.forceWalk) {
      if (threadIdx.x == 0)
        ev.sc->pixFallback = 1;
      return;
    }
    for (unsigned int j = threadIdx.x; j < n; j += blockDim.x)
      sKey[j] = ev.pixPassC[j];
    __syncthreads();
    const unsigned int plsBase = es.lsOffset[es.nLowerModules];
    Segments ls = ev.ls;
    Triplets t3 = ev.t3;
    Quintuplets t5 = ev.t5;
    for (unsigned int sIdx = threadIdx.x; sIdx < n; sIdx += blockDim.x) {
      const unsigned int key = sKey[sIdx];
      unsigned int rank = 0;
      for (unsigned int j = 0; j < n; ++j)
        rank += sKey[j] < key ? 1u : 0u;
      if (rank >= capOut)
        continue;
      const unsigned int obj = ev.pixPassObj[sIdx];
      const unsigned int iPLS = ev.pixPassPLS[sIdx];
      const float* vals = ev.pixPassV + 8 * sIdx;
      if (K == 5) {
        PT5Values v;
        v.rzChiSquared = vals[0];
        v.rPhiChiSquared = vals[1];
        v.rPhiChiSquaredInwards = vals[2];
        v.pixelRadius = vals[3];
        v.quintupletRadius = vals[4];
        v.centerX = vals[5];
        v.centerY = vals[6];
        PixelQuintuplets pt5 = ev.pt5;
        storePT5(ev.md, ls, t3, t5, pt5, plsBase + iPLS, iPLS, obj, v, rank);
      } else {
        PT3Values v;
        v.pixelRadius = vals[0];
        v.pixelRadiusError = vals[1];
        v.tripletRadius = vals[2];
        v.centerX = vals[3];
        v.centerY = vals[4];
        v.rzChiSquared = vals[5];
        v.rPhiChiSquared = vals[6];
        v.rPhiChiSquaredInwards = vals[7];
        PixelTriplets pt3 = ev.pt3;
        const short adj = es.m.layers[t3.lowerModuleIndices[3 * obj]] == 1 ? 1 : 0;
        storePT3(es.m, ev.md, ls, t3, pt3, plsBase + iPLS, iPLS, obj, adj, v, rank);
        t3.partOfPT3[obj] = 1;
      }
    }
    if (threadIdx.x == 0) {
      ev.sc->pixFallback = 0;
      const unsigned int stored = n < capOut ? n : capOut;
      if (K == 5) {
        ev.sc->nPT5Total = n;
        *ev.pt5.totOccupancyPixelQuintuplets = n;
        *ev.pt5.nPixelQuintuplets = stored;
      } else {
        ev.sc->nPT3Total = n;
        *ev.pt3.totOccupancyPixelTriplets = n;
        *ev.pt3.nPixelTriplets = stored;
      }
      if (n > capOut)
        atomicOr(&ev.sc->status, kStatusCapOverflow);
    }
  }

  // Shared pixel and outer hits of two pT3s (SDL/Kernels.h:138-200).
  // SDL/Kernels.h:325-356.  pT3 ix is removed as soon as one jx meets the
  // condition (the reference's loop breaks there), so the outcome is the OR of
  // the condition over jx: one warp per ix, its lanes over jx.
  __global__ void kPT3Dedup(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned int n = *ev.pt3.nPixelTriplets;
    PixelTriplets p = ev.pt3;
    const unsigned int wpb = blockDim.x >> 5;
    for (unsigned int ix = blockIdx.x * wpb + (threadIdx.x >> 5); ix < n; ix += gridDim.x * wpb) {
      unsigned int mine[10];
#pragma unroll
      for (int i = 0; i < 10; ++i)
        mine[i] = p.hitIndices[10 * ix + i];
      const uint8_t li = p.logicalLayers[5 * ix + 2];
      const float scoreI = p.score[ix];
      bool dup = false;
      for (unsigned int j0 = 0; j0 < n && !dup; j0 += 32) {
        const unsigned int jx = j0 + laneId();
        bool c = false;
        if (jx < n && jx != ix) {
          unsigned int other[10];
#pragma unroll
          for (int i = 0; i < 10; ++i)
            other[i] = p.hitIndices[10 * jx + i];
          int np = 0, nm = 0;
#pragma unroll
          for (int a = 0; a < 4; ++a) {
            bool m = false;
#pragma unroll
            for (int b = 0; b < 4; ++b)
              m |= mine[a] == other[b];
            np += m ? 1 : 0;
          }
#pragma unroll
          for (int a = 4; a < 10; ++a) {
            bool m = false;
#pragma unroll
            for (int b = 4; b < 10; ++b)
              m |= mine[a] == other[b];
            nm += m ? 1 : 0;
          }
          if (np + nm >= 5) {
            const uint8_t lj = p.logicalLayers[5 * jx + 2];
            const float scoreJ = p.score[jx];
            c = lj < li || (li == lj && scoreI > scoreJ) || (li == lj && scoreI == scoreJ && ix < jx);
          }
        }
        dup = __any_sync(kFullMask, c);
      }
      if (dup && laneId() == 0)
        p.isDup[ix] = 1;
    }
  }

  // ================================================== track candidates
  // pT3 vs pT5 pixel eta/phi (SDL/TrackCandidate.h:204-243).  One warp per
  // pT3, its lanes splitting the pT5 loop; the outcome is an "any" over it.
  __global__ void kCrossCleanPT3(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned int nPT3 = *ev.pt3.nPixelTriplets;
    const unsigned int nPT5 = *ev.pt5.nPixelQuintuplets;
    const unsigned int prefix = es.lsOffset[es.nLowerModules];
    const unsigned int nWarps = gridDim.x * (blockDim.x >> 5);
    for (unsigned int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < nPT3; i += nWarps) {
      if (ev.pt3.isDup[i])
        continue;
      const float eta1 = ev.pt3.eta_pix[i], phi1 = ev.pt3.phi_pix[i];
      bool dup = false;
      for (unsigned int j = laneId(); j < nPT5; j += 32) {
        unsigned int pLS_jx = ev.pt5.pixelIndices[j];
        float eta2 = ev.ls.eta[pLS_jx - prefix];
        float phi2 = ev.ls.phi[pLS_jx - prefix];
        float dEta = fabs_(eta1 - eta2);
        float dPhi = wrapDPhi(phi1, phi2);
        float dR2 = dEta * dEta + dPhi * dPhi;
        if (dR2 < 1e-5f)
          dup = true;
      }
      if (__any_sync(kFullMask, dup) && laneId() == 0)
        ev.pt3.isDup[i] = 1;
    }
  }

  // pT3 -> TC (SDL/TrackCandidate.h:383-433); one block per event.
  __global__ void __launch_bounds__(1024) kAddPT3TC(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned int n = *ev.pt3.nPixelTriplets;
    const unsigned int pLS_offset = es.lsOffset[es.nLowerModules];
    const unsigned int start = *ev.tc.nTrackCandidates;
    TrackCandidates tc = ev.tc;
    PixelTriplets p = ev.pt3;
    unsigned int carry = 0;
    for (unsigned int base = 0; base < n; base += blockDim.x) {
      unsigned int i = base + threadIdx.x;
      bool f = i < n && !p.isDup[i];
      unsigned int tot;
      unsigned int ex = blockExclusiveScan(f ? 1u : 0u, tot);
      unsigned int idx = start + carry + ex;
      if (f && idx < kMaxPixelTrackCandidates) {
        float radius = 0.5f * (p.pixelRadius[i] + p.tripletRadius[i]);
        unsigned int pix = p.pixelSegmentIndices[i];
        storeTC(tc, 5, i, i, &p.logicalLayers[5 * i], &p.lowerModuleIndices[5 * i], &p.hitIndices[10 * i],
                static_cast<int>(ev.ls.seedIdx[pix - pLS_offset]), p.centerX[i], p.centerY[i], radius, idx, i);
      }
      carry += tot;
    }
    if (threadIdx.x == 0) {
      unsigned int accepted = (start + carry <= kMaxPixelTrackCandidates) ? carry
                              : (start < kMaxPixelTrackCandidates ? kMaxPixelTrackCandidates - start : 0u);
      if (accepted < carry)
        atomicOr(&ev.sc->status, kStatusTCTruncated);
      *tc.nTrackCandidates = start + accepted;
      *tc.nTrackCandidatespT3 += accepted;
    }
  }

  // Cross-module T5 duplicate removal before TC building
  // (SDL/Kernels.h:251-323); one warp per eligible module, marks t5Flag.
  // Cross-module T5 cleaning (SDL/Kernels.h:251-323).  The reference visits
  // the ordered pairs (ix in module A, jx in module B) with A's position in
  // the eligible-module list not after B's and ix != jx; a pair whose
  // |deta| > 0.1 is skipped at the first test, and marks are only ever set.  kT5Bin counting-sorts the event's
  // quintuplets into the pLS-cleaning eta bins (one block per event), and
  // kT5DedupBinned gives each quintuplet a thread that visits the same ordered
  // pairs among the bins within reach (and the non-finite bin, which meets
  // every quintuplet, as does a quintuplet of non-finite eta).  Events with
  // more quintuplets than kT5SortCap keep the module-pair walk.
  __global__ void __launch_bounds__(1024) kT5Bin(DeviceES es, const EventView* evs) {
    __shared__ unsigned int sCount[kPLSBins + 1];
    const EventView& ev = evs[blockIdx.y];
    const int nE = *ev.rg.nEligibleT5Modules;
    const Quintuplets& q = ev.t5;
    for (int b = threadIdx.x; b <= kPLSBins; b += blockDim.x)
      sCount[b] = 0;
    __syncthreads();
    unsigned int mine = 0;
    for (int e = threadIdx.x; e < nE; e += blockDim.x) {
      const uint16_t lm = ev.rg.indicesOfEligibleT5Modules[e];
      const unsigned int n = q.nQuintuplets[lm], base = ev.rg.quintupletModuleIndices[lm];
      for (unsigned int j = 0; j < n; ++j)
        atomicAdd(&sCount[plsEtaBin(q.eta[base + j])], 1u);
      mine += n;
    }
    unsigned int total;
    blockExclusiveScan(mine, total);
    const unsigned int c = threadIdx.x <= kPLSBins ? sCount[threadIdx.x] : 0u;
    unsigned int tot;
    const unsigned int ex = blockExclusiveScan(c, tot);
    if (threadIdx.x <= kPLSBins) {
      sCount[threadIdx.x] = ex;
      ev.t5BinStart[threadIdx.x] = ex;
    }
    if (threadIdx.x == 0) {
      ev.t5BinStart[kPLSBins + 1] = tot;
      ev.sc->t5SortCount = total;
    }
    __syncthreads();
    if (total > kT5SortCap)
      return;
    for (int e = threadIdx.x; e < nE; e += blockDim.x) {
      const uint16_t lm = ev.rg.indicesOfEligibleT5Modules[e];
      const unsigned int n = q.nQuintuplets[lm], base = ev.rg.quintupletModuleIndices[lm];
      for (unsigned int j = 0; j < n; ++j) {
        const unsigned int pos = atomicAdd(&sCount[plsEtaBin(q.eta[base + j])], 1u);
        ev.t5Order[pos] = base + j;
        ev.t5OrderPos[pos] = static_cast<uint16_t>(e);
      }
    }
  }

  // The reference's test of one ordered pair (ix, jx), marking the loser.
  LST_DEV void t5CrossPair(const EventView& ev, unsigned int ix, unsigned int jx, float eta1, float phi1,
                           float score1) {
    const Quintuplets& q = ev.t5;
    if (q.partOfPT5[jx] || (q.isDup[jx] & 1))
      return;
    float eta2 = q.eta[jx], phi2 = q.phi[jx], score2 = q.score_rphisum[jx];
    float dEta = fabs_(eta1 - eta2);
    float dPhi = wrapDPhi(phi1, phi2);
    if (dEta > 0.1f)
      return;
    if (fabs_(dPhi) > 0.1f)
      return;
    float dR2 = dEta * dEta + dPhi * dPhi;
    int nMatched = sharedHitsT5(q, ix, jx);
    if (dR2 < 0.001f || nMatched >= 5) {
      if (score1 > score2)
        ev.t5Flag[ix] = 1;
      else if (score1 < score2)
        ev.t5Flag[jx] = 1;
      else
        ev.t5Flag[ix < jx ? ix : jx] = 1;
    }
  }

  __global__ void kT5DedupBinned(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned int n = ev.sc->t5SortCount;
    if (n > kT5SortCap || ev.forceWalk)
      return;
    const Quintuplets& q = ev.t5;
    const unsigned int* binStart = ev.t5BinStart;
    const unsigned int nFinite = binStart[kPLSBins];
    for (unsigned int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
      const unsigned int ix = ev.t5Order[k];
      if (q.partOfPT5[ix] || (q.isDup[ix] & 1))
        continue;
      const unsigned int posI = ev.t5OrderPos[k];
      const float eta1 = q.eta[ix], phi1 = q.phi[ix], score1 = q.score_rphisum[ix];
      const int b = plsEtaBin(eta1);
      unsigned int lo = 0, hi = n, lo2 = n;  // positions [lo, hi) then [lo2, n)
      if (b < kPLSBins) {
        lo = binStart[b >= kPLSBinReach ? b - kPLSBinReach : 0];
        hi = binStart[(b + kPLSBinReach < kPLSBins ? b + kPLSBinReach : kPLSBins - 1) + 1];
        lo2 = nFinite;
      }
      for (int part = 0; part < 2; ++part) {
        const unsigned int p0 = part == 0 ? lo : lo2, p1 = part == 0 ? hi : n;
        for (unsigned int p = p0; p < p1; ++p) {
          const unsigned int jx = ev.t5Order[p];
          const unsigned int posJ = ev.t5OrderPos[p];
          if (jx == ix || posJ < posI)
            continue;
          t5CrossPair(ev, ix, jx, eta1, phi1, score1);
        }
      }
    }
  }

  __global__ void kT5DedupBeforeTC(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    if (ev.sc->t5SortCount <= kT5SortCap && !ev.forceWalk)
      return;  // kT5DedupBinned has done this event
    // A warp per eligible module, grid-stride (the grid is kept small: most
    // events return above).
    const int nE = *ev.rg.nEligibleT5Modules;
    const int nWarps = static_cast<int>((gridDim.x * blockDim.x) >> 5);
    const Quintuplets& q = ev.t5;
    for (int warp = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5); warp < nE; warp += nWarps) {
      uint16_t lowmod1 = ev.rg.indicesOfEligibleT5Modules[warp];
      unsigned int n1 = q.nQuintuplets[lowmod1];
      unsigned int base1 = ev.rg.quintupletModuleIndices[lowmod1];
      for (unsigned int ix1 = laneId(); ix1 < n1; ix1 += 32) {
        unsigned int ix = base1 + ix1;
        if (q.partOfPT5[ix] || (q.isDup[ix] & 1))
          continue;
        float eta1 = q.eta[ix], phi1 = q.phi[ix], score1 = q.score_rphisum[ix];
        for (int idx2 = warp; idx2 < nE; idx2++) {
          uint16_t lowmod2 = ev.rg.indicesOfEligibleT5Modules[idx2];
          unsigned int n2 = q.nQuintuplets[lowmod2];
          unsigned int base2 = ev.rg.quintupletModuleIndices[lowmod2];
          for (unsigned int jx1 = 0; jx1 < n2; jx1++) {
            unsigned int jx = base2 + jx1;
            if (ix == jx)
              continue;
            if (q.partOfPT5[jx] || (q.isDup[jx] & 1))
              continue;
            float eta2 = q.eta[jx], phi2 = q.phi[jx], score2 = q.score_rphisum[jx];
            float dEta = fabs_(eta1 - eta2);
            float dPhi = wrapDPhi(phi1, phi2);
            if (dEta > 0.1f)
              continue;
            if (fabs_(dPhi) > 0.1f)
              continue;
            float dR2 = dEta * dEta + dPhi * dPhi;
            int nMatched = sharedHitsT5(q, ix, jx);
            if (dR2 < 0.001f || nMatched >= 5) {
              if (score1 > score2)
                ev.t5Flag[ix] = 1;
              else if (score1 < score2)
                ev.t5Flag[jx] = 1;
              else
                ev.t5Flag[ix < jx ? ix : jx] = 1;
            }
          }
        }
      }
    }
  }

  __global__ void kMergeT5Flag(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp >= int(*ev.rg.nEligibleT5Modules))
      return;
    uint16_t lm = ev.rg.indicesOfEligibleT5Modules[warp];
    unsigned int n = ev.t5.nQuintuplets[lm];
    unsigned int base = ev.rg.quintupletModuleIndices[lm];
    for (unsigned int j = laneId(); j < n; j += 32) {
      if (ev.t5Flag[base + j]) {
        ev.t5.isDup[base + j] |= 2;
        ev.t5Flag[base + j] = 0;
      }
    }
  }

  // T5 vs pT5/pT3 eta/phi (SDL/TrackCandidate.h:245-300); one warp per
  // eligible module, taking its T5s one after the other with the lanes
  // splitting the pT5 / pT3 loop (the outcome is an "any" over it).
  __global__ void kCrossCleanT5(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp >= int(*ev.rg.nEligibleT5Modules))
      return;
    uint16_t lm = ev.rg.indicesOfEligibleT5Modules[warp];
    unsigned int n = ev.t5.nQuintuplets[lm];
    unsigned int base = ev.rg.quintupletModuleIndices[lm];
    const unsigned int nPT5 = *ev.pt5.nPixelQuintuplets;
    const unsigned int loop_bound = nPT5 + *ev.pt3.nPixelTriplets;
    for (unsigned int j = 0; j < n; ++j) {
      const unsigned int q = base + j;
      if (ev.t5.isDup[q] or ev.t5.partOfPT5[q])
        continue;
      const float eta1 = ev.t5.eta[q], phi1 = ev.t5.phi[q];
      bool dup = false;
      for (unsigned int jx = laneId(); jx < loop_bound; jx += 32) {
        float eta2, phi2;
        if (jx < nPT5) {
          eta2 = ev.pt5.eta[jx];
          phi2 = ev.pt5.phi[jx];
        } else {
          eta2 = ev.pt3.eta[jx - nPT5];
          phi2 = ev.pt3.phi[jx - nPT5];
        }
        float dEta = fabs_(eta1 - eta2);
        float dPhi = wrapDPhi(phi1, phi2);
        float dR2 = dEta * dEta + dPhi * dPhi;
        if (dR2 < 1e-3f)
          dup = true;
      }
      if (__any_sync(kFullMask, dup) && laneId() == 0)
        ev.t5.isDup[q] = 1;
    }
  }

  // T5 -> TC (SDL/TrackCandidate.h:435-487): count per eligible module, scan,
  // then emit in (module, T5) order.
  __global__ void kT5TCCount(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp >= int(*ev.rg.nEligibleT5Modules))
      return;
    uint16_t lm = ev.rg.indicesOfEligibleT5Modules[warp];
    unsigned int n = ev.t5.nQuintuplets[lm];
    unsigned int base = ev.rg.quintupletModuleIndices[lm];
    unsigned int count = 0;
    for (unsigned int start = 0; start < n; start += 32) {
      unsigned int j = start + laneId();
      bool f = false;
      if (j < n) {
        unsigned int q = base + j;
        f = !(ev.t5.isDup[q] or ev.t5.partOfPT5[q]) && ev.t5.TightCutFlag[q];
      }
      count += __popc(__ballot_sync(kFullMask, f));
    }
    if (laneId() == 0)
      ev.moduleCount[warp] = count;
  }

  __global__ void __launch_bounds__(1024) kT5TCScan(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned int n = *ev.rg.nEligibleT5Modules;
    unsigned int carry = 0;
    for (unsigned int base = 0; base < n; base += blockDim.x) {
      unsigned int i = base + threadIdx.x;
      unsigned int c = (i < n) ? ev.moduleCount[i] : 0u;
      unsigned int tot;
      unsigned int ex = blockExclusiveScan(c, tot);
      if (i < n)
        ev.moduleOffset[i] = carry + ex;
      carry += tot;
    }
    if (threadIdx.x == 0) {
      unsigned int accepted = carry < kMaxNonPixelTrackCandidates ? carry : kMaxNonPixelTrackCandidates;
      if (accepted < carry)
        atomicOr(&ev.sc->status, kStatusTCTruncated);
      ev.moduleOffset[n] = accepted;
    }
  }

  __global__ void kT5TCEmit(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nE = *ev.rg.nEligibleT5Modules;
    if (warp >= nE)
      return;
    const unsigned int start = *ev.tc.nTrackCandidates;
    uint16_t lm = ev.rg.indicesOfEligibleT5Modules[warp];
    unsigned int n = ev.t5.nQuintuplets[lm];
    unsigned int base = ev.rg.quintupletModuleIndices[lm];
    unsigned int rank = ev.moduleOffset[warp];
    TrackCandidates tc = ev.tc;
    const Quintuplets& q = ev.t5;
    for (unsigned int s0 = 0; s0 < n; s0 += 32) {
      unsigned int j = s0 + laneId();
      bool f = false;
      unsigned int qi = base + j;
      if (j < n)
        f = !(q.isDup[qi] or q.partOfPT5[qi]) && q.TightCutFlag[qi];
      unsigned int tot;
      unsigned int r = rank + warpRank(f, tot);
      if (f && r < kMaxNonPixelTrackCandidates)
        storeTC(tc, 4, qi, qi, &q.logicalLayers[5 * qi], &q.lowerModuleIndices[5 * qi], &q.hitIndices[10 * qi], -1,
                q.regressionG[qi], q.regressionF[qi], q.regressionRadius[qi], start + r, qi);
      rank += tot;
    }
  }

  __global__ void kT5TCFinish(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    if (threadIdx.x == 0 && blockIdx.x == 0) {
      unsigned int accepted = ev.moduleOffset[*ev.rg.nEligibleT5Modules];
      *ev.tc.nTrackCandidates += accepted;
      *ev.tc.nTrackCandidatesT5 += accepted;
    }
  }

  // Per-TC record for the pLS cross-cleaning (SDL/TrackCandidate.h:302-381):
  // the candidate's type, the (eta, phi) a pLS is compared with, and the
  // four pixel hits of its pLS (pT3, pT5).
  struct TCCleanInfo {
    float eta, phi;
    int type;
    int hits[4];
  };

  LST_DEV void pixelHitsOf(const Segments& s, const MiniDoublets& md, const Hits& h, unsigned int plsIndex, int* out) {
    out[0] = static_cast<int>(h.idxs[md.anchorHitIndices[s.mdIndices[2 * plsIndex]]]);
    out[1] = static_cast<int>(h.idxs[md.anchorHitIndices[s.mdIndices[2 * plsIndex + 1]]]);
    out[2] = static_cast<int>(h.idxs[md.outerHitIndices[s.mdIndices[2 * plsIndex]]]);
    out[3] = static_cast<int>(h.idxs[md.outerHitIndices[s.mdIndices[2 * plsIndex + 1]]]);
  }

  // Shared pixel hits of two pLS (SDL/TrackCandidate.h:165-202), -1 entries skipped.
  LST_DEV int sharedPixelHits(const int* phits1, const int* phits2) {
    int npMatched = 0;
    for (int i = 0; i < 4; i++) {
      bool pmatched = false;
      if (phits1[i] == -1)
        continue;
      for (int j = 0; j < 4; j++) {
        if (phits2[j] == -1)
          continue;
        if (phits1[i] == phits2[j]) {
          pmatched = true;
          break;
        }
      }
      if (pmatched)
        npMatched++;
    }
    return npMatched;
  }

  __global__ void kTCCleanInfo(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned int nTC = *ev.tc.nTrackCandidates;
    const unsigned int prefix = es.lsOffset[es.nLowerModules];
    for (unsigned int t = blockIdx.x * blockDim.x + threadIdx.x; t < nTC; t += gridDim.x * blockDim.x) {
      TCCleanInfo info;
      info.type = ev.tc.trackCandidateType[t];
      const unsigned int innerIdx = ev.tc.objectIndices[2 * t];
      info.eta = 0.f;
      info.phi = 0.f;
      info.hits[0] = info.hits[1] = info.hits[2] = info.hits[3] = -1;
      if (info.type == 4) {
        info.eta = ev.t5.eta[innerIdx];
        info.phi = ev.t5.phi[innerIdx];
      } else if (info.type == 5) {
        info.eta = ev.pt3.eta_pix[innerIdx];
        info.phi = ev.pt3.phi_pix[innerIdx];
        pixelHitsOf(ev.ls, ev.md, ev.hits, ev.pt3.pixelSegmentIndices[innerIdx], info.hits);
      } else if (info.type == 7) {
        info.eta = ev.ls.eta[innerIdx - prefix];
        info.phi = ev.ls.phi[innerIdx - prefix];
        pixelHitsOf(ev.ls, ev.md, ev.hits, innerIdx, info.hits);
      }
      ev.tcCleanInfo[t] = info;
    }
  }

  // pLS vs existing TCs (SDL/TrackCandidate.h:302-381).  A quadruplet pLS
  // that is not yet a duplicate becomes one if some TC of type 5 or 7 shares a
  // pixel hit with it, if some T5 TC (type 4) lies within dR^2 < 1e-3, or if
  // some type 5 / 7 TC lies within dR^2 < 1e-6; the outcome is an OR over the
  // TCs, so it is evaluated per pLS without walking every TC:
  //  - the pixel hits of all type 5 / 7 TCs go into a shared-memory hash set,
  //    and a pLS shares a hit with one of them iff one of its hits is in it;
  //  - the TCs are counting-sorted by eta into the pLS-cleaning bins (width
  //    0.02), and only bins within kXCleanReach of the pLS's bin are read:
  //    dR^2 < 1e-3 needs |deta| < 0.0317 (two bin widths plus rounding), and a
  //    non-finite eta or dR^2 never passes the test.
  // A set with more TCs than kXCleanMaxTC, or more hits than the hash holds,
  // is checked pair by pair instead.
  constexpr unsigned int kXCleanHashSlots = 1u << 14;
  constexpr unsigned int kXCleanMaxTC = 4096;
  constexpr int kXCleanReach = 3;
  constexpr int kXCleanBlocksPerEvent = 4;
  constexpr size_t kXCleanSmem =
      kXCleanHashSlots * 4 + 2 * (kPLSBins + 2) * 4 + kXCleanMaxTC * (sizeof(float) * 2 + sizeof(int));

  LST_DEV unsigned int xcleanSlot(unsigned int key) { return (key * 2654435761u) >> 18; }

  LST_DEV bool xcleanPairDup(const TCCleanInfo& info, const int* phits1, float eta1, float phi1) {
    if (info.type == 4) {
      float dEta = fabs_(eta1 - info.eta);
      float dPhi = wrapDPhi(phi1, info.phi);
      return dEta * dEta + dPhi * dPhi < 1e-3f;
    }
    if (info.type == 5 || info.type == 7) {
      if (sharedPixelHits(phits1, info.hits) > 0)
        return true;
      float dEta = fabs_(eta1 - info.eta);
      float dPhi = wrapDPhi(phi1, info.phi);
      return dEta * dEta + dPhi * dPhi < 0.000001f;
    }
    return false;
  }

  __global__ void __launch_bounds__(1024) kCrossCleanPLS(DeviceES es, const EventView* evs) {
    extern __shared__ __align__(16) unsigned char xsm[];
    unsigned int* sHash = reinterpret_cast<unsigned int*>(xsm);
    unsigned int* sBinStart = sHash + kXCleanHashSlots;
    unsigned int* sCursor = sBinStart + kPLSBins + 2;
    float* sEta = reinterpret_cast<float*>(sCursor + kPLSBins + 2);
    float* sPhi = sEta + kXCleanMaxTC;
    int* sType = reinterpret_cast<int*>(sPhi + kXCleanMaxTC);
    __shared__ unsigned int sOverflow;
    const EventView& ev = evs[blockIdx.y];
    const unsigned int nPix = ev.ls.nSegments[es.pixelModule];
    const unsigned int prefix = es.lsOffset[es.nLowerModules];
    const unsigned int nTC = *ev.tc.nTrackCandidates;
    const TCCleanInfo* infos = ev.tcCleanInfo;
    Segments s = ev.ls;

    if (threadIdx.x == 0)
      sOverflow = (nTC > kXCleanMaxTC || ev.forceWalk) ? 1u : 0u;
    for (unsigned int t = threadIdx.x; t < kXCleanHashSlots; t += blockDim.x)
      sHash[t] = 0;
    for (unsigned int t = threadIdx.x; t < kPLSBins + 2; t += blockDim.x)
      sCursor[t] = 0;
    __syncthreads();
    const bool fits = nTC <= kXCleanMaxTC;
    if (fits) {
      for (unsigned int t = threadIdx.x; t < nTC; t += blockDim.x) {
        const TCCleanInfo info = infos[t];
        if (info.type == 5 || info.type == 7) {
          for (int a = 0; a < 4; ++a) {
            if (info.hits[a] == -1)
              continue;
            const unsigned int key = static_cast<unsigned int>(info.hits[a]) + 1u;
            unsigned int slot = xcleanSlot(key), probes = 0;
            while (true) {
              const unsigned int old = atomicCAS(&sHash[slot], 0u, key);
              if (old == 0u || old == key)
                break;
              if (++probes == kXCleanHashSlots) {
                sOverflow = 1;
                break;
              }
              slot = (slot + 1) & (kXCleanHashSlots - 1);
            }
          }
        }
        if (info.type == 4 || info.type == 5 || info.type == 7)
          atomicAdd(&sCursor[plsEtaBin(info.eta)], 1u);
      }
    }
    __syncthreads();
    const bool fast = sOverflow == 0;
    if (fast) {
      unsigned int tot;
      const unsigned int c = threadIdx.x <= kPLSBins ? sCursor[threadIdx.x] : 0u;
      const unsigned int ex = blockExclusiveScan(c, tot);
      if (threadIdx.x <= kPLSBins) {
        sBinStart[threadIdx.x] = ex;
        sCursor[threadIdx.x] = ex;
      }
      if (threadIdx.x == 0)
        sBinStart[kPLSBins + 1] = tot;
      __syncthreads();
      for (unsigned int t = threadIdx.x; t < nTC; t += blockDim.x) {
        const TCCleanInfo& info = infos[t];
        if (info.type == 4 || info.type == 5 || info.type == 7) {
          const unsigned int pos = atomicAdd(&sCursor[plsEtaBin(info.eta)], 1u);
          sEta[pos] = info.eta;
          sPhi[pos] = info.phi;
          sType[pos] = info.type;
        }
      }
      __syncthreads();
    }

    for (unsigned int i = blockIdx.x * blockDim.x + threadIdx.x; i < nPix; i += gridDim.x * blockDim.x) {
      if (!s.isQuad[i] || s.isDup[i])
        continue;
      int phits1[4];
      pixelHitsOf(s, ev.md, ev.hits, prefix + i, phits1);
      const float eta1 = s.eta[i], phi1 = s.phi[i];
      bool dup = false;
      if (fast) {
        for (int a = 0; a < 4 && !dup; ++a) {
          if (phits1[a] == -1)
            continue;
          const unsigned int key = static_cast<unsigned int>(phits1[a]) + 1u;
          unsigned int slot = xcleanSlot(key);
          for (unsigned int probes = 0; probes < kXCleanHashSlots; ++probes) {
            const unsigned int h = sHash[slot];
            if (h == key) {
              dup = true;
              break;
            }
            if (h == 0u)
              break;
            slot = (slot + 1) & (kXCleanHashSlots - 1);
          }
        }
        const int b = plsEtaBin(eta1);
        if (!dup && b < kPLSBins) {
          const int b0 = b >= kXCleanReach ? b - kXCleanReach : 0;
          const int b1 = b + kXCleanReach < kPLSBins ? b + kXCleanReach : kPLSBins - 1;
          for (unsigned int k = sBinStart[b0]; k < sBinStart[b1 + 1] && !dup; ++k) {
            float dEta = fabs_(eta1 - sEta[k]);
            float dPhi = wrapDPhi(phi1, sPhi[k]);
            const float dR2 = dEta * dEta + dPhi * dPhi;
            dup = sType[k] == 4 ? dR2 < 1e-3f : dR2 < 0.000001f;
          }
        }
      } else {
        for (unsigned int t = 0; t < nTC && !dup; ++t)
          dup = xcleanPairDup(infos[t], phits1, eta1, phi1);
      }
      if (dup)
        s.isDup[i] = 1;
    }
  }

  __global__ void __launch_bounds__(1024) kAddPLSTC(DeviceES es, const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned int n = ev.ls.nSegments[es.pixelModule];
    const unsigned int start = *ev.tc.nTrackCandidates;
    const unsigned int nT5TC = *ev.tc.nTrackCandidatesT5;
    TrackCandidates tc = ev.tc;
    const Segments& s = ev.ls;
    unsigned int carry = 0;
    for (unsigned int base = 0; base < n; base += blockDim.x) {
      unsigned int i = base + threadIdx.x;
      bool f = i < n && s.isQuad[i] && !s.isDup[i];
      unsigned int tot;
      unsigned int ex = blockExclusiveScan(f ? 1u : 0u, tot);
      unsigned int idx = start + carry + ex;
      if (f && idx - nT5TC < kMaxPixelTrackCandidates) {
        tc.trackCandidateType[idx] = 8;
        tc.directObjectIndices[idx] = i;
        tc.pixelSeedIndex[idx] = static_cast<int>(s.seedIdx[i]);
        tc.objectIndices[2 * idx] = i;
        tc.objectIndices[2 * idx + 1] = i;
        tc.hitIndices[14 * idx + 0] = s.pLSHitsIdxs[4 * i + 0];
        tc.hitIndices[14 * idx + 1] = s.pLSHitsIdxs[4 * i + 2];
        tc.hitIndices[14 * idx + 2] = s.pLSHitsIdxs[4 * i + 1];
        tc.hitIndices[14 * idx + 3] = s.pLSHitsIdxs[4 * i + 3];
        for (int k = 4; k < 14; ++k)
          tc.hitIndices[14 * idx + k] = 0;
        for (int k = 0; k < 7; ++k) {
          tc.logicalLayers[7 * idx + k] = 0;
          tc.lowerModuleIndices[7 * idx + k] = 0;
        }
        tc.centerX[idx] = 0;
        tc.centerY[idx] = 0;
        tc.radius[idx] = 0;
      }
      carry += tot;
    }
    if (threadIdx.x == 0) {
      unsigned int room = (start - nT5TC < kMaxPixelTrackCandidates) ? kMaxPixelTrackCandidates - (start - nT5TC) : 0u;
      unsigned int accepted = carry < room ? carry : room;
      if (accepted < carry)
        atomicOr(&ev.sc->status, kStatusTCTruncated);
      *tc.nTrackCandidates = start + accepted;
      *tc.nTrackCandidatespLS += accepted;
    }
  }


  // ============================================================== counts
  // Object counts of one event, as the reference's getNumberOf* members
  // (SDL/Event.cc:1148-1487): per-layer sums over lower modules with the
  // same inclusion rules as add*ToEventExplicit.  One block per event.
  __global__ void kCounts(DeviceES es, const EventView* evs) {
    __shared__ unsigned int sBins[4][11];
    const EventView& ev = evs[blockIdx.y];
    for (int i = threadIdx.x; i < 44; i += blockDim.x)
      (&sBins[0][0])[i] = 0;
    __syncthreads();
    const Modules& m = es.m;
    for (unsigned int i = threadIdx.x; i < es.nLowerModules; i += blockDim.x) {
      int bin = (m.subdets[i] == Barrel) ? (m.layers[i] - 1) : (6 + m.layers[i] - 1);
      if (bin < 0 || bin >= 11)
        continue;
      unsigned int nmd = ev.md.nMDs[i];
      if (!(nmd == 0 or ev.hits.hitRanges[i * 2] == -1))
        atomicAdd(&sBins[0][bin], nmd);
      unsigned int nls = ev.ls.nSegments[i];
      if (nls != 0)
        atomicAdd(&sBins[1][bin], nls);
      unsigned int nt3 = ev.t3.nTriplets[i];
      if (nt3 != 0)
        atomicAdd(&sBins[2][bin], nt3);
      unsigned int nt5 = ev.t5.nQuintuplets[i];
      if (!(nt5 == 0 or ev.rg.quintupletModuleIndices[i] == -1))
        atomicAdd(&sBins[3][bin], nt5);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      lst_counts* c = ev.counts;
      c->nHits = ev.sc->nHits;
      c->nPixelSegments = ev.ls.nSegments[es.pixelModule];
      c->status = ev.sc->status;
      unsigned int tot[4] = {0, 0, 0, 0};
      for (int k = 0; k < 4; ++k)
        for (int b = 0; b < 11; ++b)
          tot[k] += sBins[k][b];
      for (int b = 0; b < 6; ++b) {
        c->mdBarrel[b] = sBins[0][b];
        c->lsBarrel[b] = sBins[1][b];
        c->t3Barrel[b] = sBins[2][b];
        c->t5Barrel[b] = sBins[3][b];
      }
      for (int b = 0; b < 5; ++b) {
        c->mdEndcap[b] = sBins[0][6 + b];
        c->lsEndcap[b] = sBins[1][6 + b];
        c->t3Endcap[b] = sBins[2][6 + b];
        c->t5Endcap[b] = sBins[3][6 + b];
      }
      c->nMiniDoublets = tot[0];
      c->nSegments = tot[1];
      c->nTriplets = tot[2];
      c->nQuintuplets = tot[3];
      c->nPixelTriplets = *ev.pt3.nPixelTriplets;
      c->nPixelQuintuplets = *ev.pt5.nPixelQuintuplets;
      c->nTrackCandidates = *ev.tc.nTrackCandidates;
      c->nTrackCandidatesPT5 = *ev.tc.nTrackCandidatespT5;
      c->nTrackCandidatesPT3 = *ev.tc.nTrackCandidatespT3;
      c->nTrackCandidatesPLS = *ev.tc.nTrackCandidatespLS;
      c->nTrackCandidatesT5 = *ev.tc.nTrackCandidatesT5;
      c->nPixelTripletsFound = ev.sc->nPT3Total;
      c->nPixelQuintupletsFound = ev.sc->nPT5Total;
      for (int k = 0; k < 4; ++k)
        c->reserved[k] = 0;
    }
  }

  // ============================================================ inputs
  // Sets the hit and pLS counts of one event (per-event input path).
  __global__ void kSetInputCounts(const EventView* evs, int slot, int setHits, unsigned int nHits, int setPLS,
                                  unsigned int nPLS, unsigned int statusBits) {
    const EventView& ev = evs[slot];
    if (setHits)
      ev.sc->nHits = nHits;
    if (setPLS)
      ev.sc->nPLS = nPLS;
    ev.sc->status |= statusBits;
  }

  // Byte layout of one packed input event (see lst_packed_size).
  struct PackedLayout {
    size_t x, y, z, detId, idx, h0, h1, h2, h3, dPhiChange, ptIn, ptErr, px, py, pz, eta, etaErr, phi, charge,
        seedIdx, superbin, pixelType, isQuad, end;
  };
  LST_HD PackedLayout packedLayout(unsigned int nHits, unsigned int nPLS) {
    PackedLayout L;
    size_t o = 16;
    size_t h4 = 4 * size_t(nHits), p4 = 4 * size_t(nPLS);
    L.x = o; o += h4;
    L.y = o; o += h4;
    L.z = o; o += h4;
    L.detId = o; o += h4;
    L.idx = o; o += h4;
    L.h0 = o; o += p4;
    L.h1 = o; o += p4;
    L.h2 = o; o += p4;
    L.h3 = o; o += p4;
    L.dPhiChange = o; o += p4;
    L.ptIn = o; o += p4;
    L.ptErr = o; o += p4;
    L.px = o; o += p4;
    L.py = o; o += p4;
    L.pz = o; o += p4;
    L.eta = o; o += p4;
    L.etaErr = o; o += p4;
    L.phi = o; o += p4;
    L.charge = o; o += p4;
    L.seedIdx = o; o += p4;
    L.superbin = o; o += p4;
    L.pixelType = o; o += nPLS;
    L.isQuad = o; o += nPLS;
    L.end = (o + 15) & ~size_t(15);
    return L;
  }

  // Unpacks the packed inputs of a batch into the event stores: the hits
  // (addHitToEvent's copies) and the pixel-segment fields
  // (addPixelSegmentToEvent's copies).  blockIdx.y = event within the batch.
  __global__ void kUnpack(const EventView* evs, const unsigned char* blobs, const unsigned long long* offsets,
                          unsigned long long totalBytes) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned char* b = blobs + offsets[blockIdx.y];
    const unsigned int* hdr = reinterpret_cast<const unsigned int*>(b);
    unsigned int nHits = hdr[0], nPLSIn = hdr[1];
    unsigned int status = 0;
    // A blob whose arrays would end beyond the uploaded bytes is dropped.
    const bool truncated = offsets[blockIdx.y] + packedLayout(nHits, nPLSIn).end > totalBytes;
    if (truncated) {
      status |= kStatusInvalidInput;
      nHits = 0;
      nPLSIn = 0;
    }
    bool reject = nHits > ev.maxHits;
    unsigned int nPLS = nPLSIn;
    if (reject) {
      status |= kStatusHitCapacity;
      nHits = 0;
      nPLS = 0;
    }
    if (nPLS > kMaxPixelSegments) {
      status |= kStatusPLSTruncated;
      nPLS = kMaxPixelSegments;
    }
    if (nHits == 0 && nPLS > 0) {
      status |= kStatusInvalidInput;
      nPLS = 0;
    }
    const PackedLayout L = packedLayout(reject ? 0u : nHits, reject ? 0u : nPLSIn);
    const unsigned int stride = gridDim.x * blockDim.x;
    const unsigned int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    // Two hits per thread and step: ten loads in flight before the stores.
    for (unsigned int i = t0; i < nHits; i += 2 * stride) {
      const unsigned int j = i + stride;
      const bool two = j < nHits;
      const float x0 = reinterpret_cast<const float*>(b + L.x)[i];
      const float y0 = reinterpret_cast<const float*>(b + L.y)[i];
      const float z0 = reinterpret_cast<const float*>(b + L.z)[i];
      const unsigned int d0 = reinterpret_cast<const unsigned int*>(b + L.detId)[i];
      const unsigned int n0 = reinterpret_cast<const unsigned int*>(b + L.idx)[i];
      float x1 = 0.f, y1 = 0.f, z1 = 0.f;
      unsigned int d1 = 0, n1 = 0;
      if (two) {
        x1 = reinterpret_cast<const float*>(b + L.x)[j];
        y1 = reinterpret_cast<const float*>(b + L.y)[j];
        z1 = reinterpret_cast<const float*>(b + L.z)[j];
        d1 = reinterpret_cast<const unsigned int*>(b + L.detId)[j];
        n1 = reinterpret_cast<const unsigned int*>(b + L.idx)[j];
      }
      ev.hits.xs[i] = x0;
      ev.hits.ys[i] = y0;
      ev.hits.zs[i] = z0;
      ev.hits.detid[i] = d0;
      ev.hits.idxs[i] = n0;
      if (two) {
        ev.hits.xs[j] = x1;
        ev.hits.ys[j] = y1;
        ev.hits.zs[j] = z1;
        ev.hits.detid[j] = d1;
        ev.hits.idxs[j] = n1;
      }
    }
    for (unsigned int i = t0; i < nPLS; i += stride) {
      ev.plsHit0[i] = reinterpret_cast<const unsigned int*>(b + L.h0)[i];
      ev.plsHit1[i] = reinterpret_cast<const unsigned int*>(b + L.h1)[i];
      ev.plsHit2[i] = reinterpret_cast<const unsigned int*>(b + L.h2)[i];
      ev.plsHit3[i] = reinterpret_cast<const unsigned int*>(b + L.h3)[i];
      ev.plsDPhiChange[i] = reinterpret_cast<const float*>(b + L.dPhiChange)[i];
      ev.ls.ptIn[i] = reinterpret_cast<const float*>(b + L.ptIn)[i];
      ev.ls.ptErr[i] = reinterpret_cast<const float*>(b + L.ptErr)[i];
      ev.ls.px[i] = reinterpret_cast<const float*>(b + L.px)[i];
      ev.ls.py[i] = reinterpret_cast<const float*>(b + L.py)[i];
      ev.ls.pz[i] = reinterpret_cast<const float*>(b + L.pz)[i];
      ev.ls.eta[i] = reinterpret_cast<const float*>(b + L.eta)[i];
      ev.ls.etaErr[i] = reinterpret_cast<const float*>(b + L.etaErr)[i];
      ev.ls.phi[i] = reinterpret_cast<const float*>(b + L.phi)[i];
      ev.ls.charge[i] = reinterpret_cast<const int*>(b + L.charge)[i];
      ev.ls.seedIdx[i] = reinterpret_cast<const unsigned int*>(b + L.seedIdx)[i];
      ev.ls.superbin[i] = reinterpret_cast<const int*>(b + L.superbin)[i];
      ev.ls.pixelType[i] = reinterpret_cast<const int8_t*>(b + L.pixelType)[i];
      ev.ls.isQuad[i] = reinterpret_cast<const int8_t*>(b + L.isQuad)[i];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      ev.sc->nHits = nHits;
      ev.sc->nPLS = nPLS;
      ev.sc->status |= status;
    }
  }


  // ============================================================ output
  // Track-candidate output in the form of LST::getOutput
  // (SDL/LST.cc:367-427): per candidate its type, pixel seed index and the
  // list of input-ntuple hit indices (14 / 10 / 10 / 4 slots for pT5 / pT3 /
  // T5 / pLS, a repeated 4th hit of pixel objects dropped).
  __device__ __forceinline__ int tcOutputHits(const EventView& ev, unsigned int idx, unsigned int* out) {
    const short type = ev.tc.trackCandidateType[idx];
    const int maxN = type == 7 ? 14 : (type == 5 ? 10 : (type == 4 ? 10 : (type == 8 ? 4 : 0)));
    int n = 0;
    unsigned int last = 0;
    for (int i = 0; i < maxN; ++i) {
      unsigned int g = ev.tc.hitIndices[14 * idx + i];
      unsigned int h = (type == 8) ? g : ev.hits.idxs[g];
      if (type != 4 && n == 3 && last == h)
        continue;
      if (out)
        out[n] = h;
      ++n;
      last = h;
    }
    return n;
  }

  // Per event: output length of every candidate and their offsets; one block
  // per event.
  __global__ void __launch_bounds__(1024) kOutputSizes(const EventView* evs) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned int n = *ev.tc.nTrackCandidates;
    unsigned int carry = 0;
    for (unsigned int base = 0; base < n; base += blockDim.x) {
      unsigned int i = base + threadIdx.x;
      unsigned int len = (i < n) ? static_cast<unsigned int>(tcOutputHits(ev, i, nullptr)) : 0u;
      unsigned int tot;
      unsigned int ex = blockExclusiveScan(len, tot);
      if (i < n) {
        ev.tcOutLen[i] = len;
        ev.tcOutOffset[i] = carry + ex;
      }
      carry += tot;
    }
    if (threadIdx.x == 0)
      ev.sc->nOutHits = carry;
  }

  // Offsets of each event's candidates and hits inside the batch output
  // (exclusive scans over the events); one block.
  __global__ void __launch_bounds__(1024) kOutputEventOffsets(const EventView* evs, int count,
                                                              unsigned long long* offsets) {
    unsigned long long carryTC = 0, carryHits = 0;
    for (int base = 0; base < count; base += blockDim.x) {
      int i = base + threadIdx.x;
      unsigned int ntc = (i < count) ? *evs[i].tc.nTrackCandidates : 0u;
      unsigned int nh = (i < count) ? evs[i].sc->nOutHits : 0u;
      unsigned int totTC, totH;
      unsigned int exTC = blockExclusiveScan(ntc, totTC);
      unsigned int exH = blockExclusiveScan(nh, totH);
      if (i < count) {
        offsets[i] = carryTC + exTC;
        offsets[count + 1 + i] = carryHits + exH;
      }
      carryTC += totTC;
      carryHits += totH;
    }
    if (threadIdx.x == 0) {
      offsets[count] = carryTC;
      offsets[2 * count + 1] = carryHits;
    }
  }

  // Writes the batch output: hits, len, seedIdx and type, contiguous.
  __global__ void kOutputGather(const EventView* evs, int count, const unsigned long long* offsets,
                                unsigned int* outHits, unsigned int* outLen, int* outSeed, short* outType) {
    const EventView& ev = evs[blockIdx.y];
    const unsigned int n = *ev.tc.nTrackCandidates;
    const unsigned long long tc0 = offsets[blockIdx.y];
    const unsigned long long h0 = offsets[count + 1 + blockIdx.y];
    for (unsigned int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
      tcOutputHits(ev, i, outHits + h0 + ev.tcOutOffset[i]);
      outLen[tc0 + i] = ev.tcOutLen[i];
      outSeed[tc0 + i] = ev.tc.pixelSeedIndex[i];
      outType[tc0 + i] = ev.tc.trackCandidateType[i];
    }
  }

}  // namespace lst

#include "lst_seed.h"
