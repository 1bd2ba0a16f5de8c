// Device-side views of the event setup and of one event's object stores.
#pragma once

#include "lst_b200.h"
#include "lst_pixel.h"

namespace lst {

  struct TCCleanInfo;
  struct PLSRec;

  // Event setup resident on the device (read-only during an event).
  struct DeviceES {
    Modules m;
    const unsigned int* cpIndex;
    const unsigned int* cpSizes;
    const unsigned int* cpIndexPos;
    const unsigned int* cpSizesPos;
    const unsigned int* cpIndexNeg;
    const unsigned int* cpSizesNeg;
    unsigned int pixelIndexOffsetPos;
    unsigned int pixelIndexOffsetNeg;
    const int* mdOffset;
    const int* mdCap;
    const int* lsOffset;
    const int* lsCap;
    const int* t3CapIfUsed;
    const int* t5CapIfEligible;
    unsigned int nTotalMDs;
    unsigned int nTotalSegments;
    unsigned int maxTriplets;
    unsigned int maxQuintuplets;
    const unsigned int* detHashKey;
    const uint16_t* detHashVal;
    unsigned int detHashBits;
    uint16_t nModules;
    uint16_t nLowerModules;
    uint16_t pixelModule;
  };

  // Status bits reported per event.
  enum StatusBits : unsigned int {
    kStatusUnknownDetId = 1u << 0,       // a hit's detId is not in the geometry
    kStatusUnknownEndcapDetId = 1u << 1,  // a 2S endcap hit without strip orientation
    kStatusHitCapacity = 1u << 2,        // more hits than the event store holds
    kStatusPLSTruncated = 1u << 3,       // more than 50000 pLS: the rest were dropped (as the reference does)
    kStatusTCTruncated = 1u << 4,        // a track-candidate cap was reached
    kStatusCapOverflow = 1u << 5,        // an occupancy cap dropped objects (as the reference does)
    kStatusInvalidInput = 1u << 6,       // a pLS hit index beyond the event's hits (replaced by hit 0)
  };

  // Per-event scalars in device memory.
  struct EventScalars {
    unsigned int nHits;
    unsigned int nPLS;
    unsigned int status;
    unsigned int nPT5Total;
    unsigned int nPT3Total;
    unsigned int nOutHits;  // output hit-list length of the event's track candidates
    unsigned int t5CandTotal;     // quintuplet candidates of the event
    unsigned int t5CandOverflow;  // more candidates than the flag buffer holds
    unsigned int t5PassCount;     // passing candidates found by kT5Eval
    unsigned int pixCandTotal;    // pT5 / pT3 candidates of the current pixel stage
    unsigned int pixPassCount;    // passing candidates found by kPixEval
    unsigned int pixFallback;     // the pixel stage overflowed the staging: walk instead
    unsigned int pixQueueCount;   // candidates passing the pixel pre-selection
    unsigned int t5QueueCount;    // candidates passing the quintuplet pre-selection
    unsigned int pixQueueBack;    // pixel candidates queued from the back (endcap tracklet algorithm)
    unsigned int t5QueueBack;     // quintuplet candidates queued from the back (modules not all barrel)
    unsigned int pixQueue2Count;  // pixel candidates passing the first pixel tracklet as well
    unsigned int t5SortCount;     // quintuplets binned by eta for the cross-module cleaning
    unsigned int mdNext;          // next task for kCreateMD's warps
    unsigned int lsNext;          // next lower module for kCreateLS's warps
    unsigned int t3Next;          // next lower module for kCreateT3's warps
  };

  // All device pointers of one event.
  struct EventView {
    Hits hits;
    Ranges rg;
    MiniDoublets md;
    Segments ls;
    Triplets t3;
    Quintuplets t5;
    PixelTriplets pt3;
    PixelQuintuplets pt5;
    TrackCandidates tc;
    EventScalars* sc;
    lst_counts* counts;
    // pLS inputs that are not stored in the segment store
    unsigned int* plsHit0;
    unsigned int* plsHit1;
    unsigned int* plsHit2;
    unsigned int* plsHit3;
    float* plsDPhiChange;
    // scratch
    unsigned int* plsConnIndex;
    unsigned int* plsConnSize;
    unsigned int* plsCount;
    unsigned int* plsOffset;
    unsigned int* moduleCount;
    unsigned int* moduleOffset;
    uint8_t* t5Flag;   // removal marks of the cross-module T5 cleaning
    uint8_t* plsFlag;  // removal marks of the second pLS cleaning pass
    unsigned int* tcOutLen;     // output hits per track candidate
    unsigned int* tcOutOffset;  // offset of a candidate's hits in the event's output
    // MD-keyed indices: per module, segments / triplets grouped by their first
    // MD (module-relative indices), with per-MD start and count
    uint16_t* lsByMD;
    uint16_t* mdLSStart;
    uint16_t* mdLSCount;
    uint16_t* t3ByMD;
    uint16_t* mdT3Start;
    uint16_t* mdT3Count;
    unsigned int* t5CandPre;    // per inner triplet: its first candidate within the module
    unsigned int* t5ModCand;    // per eligible module: candidates
    unsigned int* t5ModOff;     // per eligible module: first candidate of the event
    unsigned int* t5CandFlag;   // per candidate: 0 = fails, else 1 + slot of its values in t5PassValues
    T5Values* t5PassValues;     // selection values of passing candidates
    unsigned int* t5PassC;      //   and their candidate index
    float* t5DnnFeat;           // candidates staged for the classifier (kT5Eval): 38 inputs each
    struct T5DnnSlotG* t5DnnSlot;  //   and their selection state
    unsigned int* plsModPre;    // per pLS: candidate prefix over its connected modules (41 entries)
    unsigned int* plsCand;      // per pLS: candidates
    unsigned int* plsCandOff;   // per pLS: first candidate (nPLS + 1 entries)
    unsigned int* pixPassC;     // passing candidates: candidate index
    unsigned int* pixPassObj;   //   the T5 / T3 index
    unsigned int* pixPassPLS;   //   the pLS index
    float* pixPassV;            //   the selection values (8 per candidate)
    float* hitMiniSlope;        // per hit: the slope term of the mini-doublet dphi threshold
    float* hitShiftXa;          // per hit moved by the strip shift: its moved point and z
    float* hitShiftYa;
    float* hitShiftZn;
    unsigned int* t5Order;      // quintuplets sorted by eta bin (their index)
    uint16_t* t5OrderPos;       //   and their module's position in the eligible-module list
    unsigned int* t5BinStart;   // start of each eta bin in t5Order (bins + 2 entries)
    unsigned int* candQueue;    // candidates passing a pre-selection (T5, then pT5 / pT3), any order
    unsigned int* pixChunkPLS;  // per 32 pT5 / pT3 candidates: the pLS of the first one
    unsigned int* t5ChunkMod;   // per 32 T5 candidates: the eligible module of the first one
    struct TCCleanInfo* tcCleanInfo;  // per track candidate: the pLS cross-cleaning record
    struct PLSRec* plsRec;      // pass-2 pLS records sorted by eta bin
    unsigned int* plsHitHead;   // hit -> pLS index of the pLS cleaning: chain head per bucket
    unsigned int* plsHitNext;   //   and the next entry (4 pLS + hit slot) per entry
    unsigned int* plsBinStart;  // start of each eta bin in plsRec (bins + 2 entries)
    unsigned int maxHits;
    unsigned int forceWalk;  // take the fallback paths (walks, pair-by-pair tests) for testing them
  };

}  // namespace lst
