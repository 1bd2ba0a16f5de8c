/* C ABI of the B200 LST object-building chain (hits -> mini-doublets ->
 * line segments -> triplets -> quintuplets -> pixel triplets/quintuplets ->
 * track candidates).
 *
 * The reference exposes this path only as C++ classes templated on Alpaka
 * types: SDL::Event<Acc> (SDL/Event.h:31-205, SDL/Event.cc) and the
 * event-setup loaders (SDL/LSTESData.h:79-80).  Each entry point below states
 * the reference member it replaces.  Conventions:
 *   - every function returns an int status: 0 = ok, < 0 = error (the message
 *     is available from lst_last_error()), > 0 = the event's status bits
 *     (LST_STATUS_*) where a function reports them;
 *   - no C++ exceptions cross this boundary;
 *   - a handle is used by one host thread at a time; an event set owns its
 *     CUDA stream (or borrows the caller's) and all its device memory;
 *   - an event setup (lst_es) is read-only once loaded and may be shared by
 *     any number of event sets on the same device.
 *
 * Event sets hold N event slots.  The per-event calls take a slot index and
 * behave as the matching SDL::Event member on that event.  The batched calls
 * (lst_batch_*) run a stage for slots [first, first + count) in one launch per
 * kernel.
 */
#ifndef LST_B200_H
#define LST_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lst_es lst_es;
typedef struct lst_event lst_event;

/* Status bits an event can report (returned by stage calls and in counts). */
#define LST_STATUS_UNKNOWN_DETID 0x1u        /* a hit's detId is not in the geometry */
#define LST_STATUS_UNKNOWN_ENDCAP_DETID 0x2u /* 2S endcap hit without strip orientation */
#define LST_STATUS_HIT_CAPACITY 0x4u         /* more hits than the slot holds: event rejected */
#define LST_STATUS_PLS_TRUNCATED 0x8u        /* more than 50000 pLS: the rest dropped (as the reference) */
#define LST_STATUS_TC_TRUNCATED 0x10u        /* a track-candidate cap was reached (as the reference) */
#define LST_STATUS_CAP_OVERFLOW 0x20u        /* an occupancy cap dropped objects (as the reference) */
#define LST_STATUS_INVALID_INPUT 0x40u       /* a pLS hit index >= nHits (replaced by hit 0), or pLS without hits */

/* Stage identifiers for lst_batch_run / lst_event_run_stage. */
enum lst_stage {
  LST_STAGE_MINI_DOUBLETS = 1,     /* Event::createMiniDoublets            SDL/Event.cc:393 */
  LST_STAGE_SEGMENTS = 2,          /* Event::createSegmentsWithModuleMap   SDL/Event.cc:469 */
  LST_STAGE_TRIPLETS = 3,          /* Event::createTriplets                SDL/Event.cc:512 */
  LST_STAGE_QUINTUPLETS = 4,       /* Event::createQuintuplets             SDL/Event.cc:903 */
  LST_STAGE_PLS_CLEANING = 5,      /* Event::pixelLineSegmentCleaning      SDL/Event.cc:993 */
  LST_STAGE_PIXEL_QUINTUPLETS = 6, /* Event::createPixelQuintuplets        SDL/Event.cc:1009 */
  LST_STAGE_PIXEL_TRIPLETS = 7,    /* Event::createPixelTriplets           SDL/Event.cc:784 */
  LST_STAGE_TRACK_CANDIDATES = 8   /* Event::createTrackCandidates         SDL/Event.cc:620 */
};

/* T5 selection method used by LST_STAGE_QUINTUPLETS. */
enum lst_t5_method {
  LST_T5_DNN = 0,     /* reference default: rz chi2 + DNN (USE_RZCHI2, USE_T5_DNN) */
  LST_T5_CUTS = 1     /* cut-only: rz chi2 + r-phi chi2 (USE_RZCHI2, USE_RPHICHI2) */
};

/* Object counts of one event (SDL/Event.cc:1263-1487 getNumberOf*). */
typedef struct lst_counts {
  uint32_t nHits;
  uint32_t nPixelSegments;
  uint32_t status;
  uint32_t nMiniDoublets;     /* summed over lower modules, as getNumberOfMiniDoublets */
  uint32_t nSegments;         /* as getNumberOfSegments */
  uint32_t nTriplets;         /* as getNumberOfTriplets */
  uint32_t nQuintuplets;      /* as getNumberOfQuintuplets */
  uint32_t nPixelTriplets;    /* as getNumberOfPixelTriplets (stored, <= 5000) */
  uint32_t nPixelQuintuplets; /* as getNumberOfPixelQuintuplets (stored, <= 15000) */
  uint32_t nTrackCandidates;
  uint32_t nTrackCandidatesPT5;
  uint32_t nTrackCandidatesPT3;
  uint32_t nTrackCandidatesPLS;
  uint32_t nTrackCandidatesT5;
  uint32_t nPixelTripletsFound;    /* before the 5000 cap */
  uint32_t nPixelQuintupletsFound; /* before the 15000 cap */
  uint32_t mdBarrel[6], mdEndcap[5]; /* getNumberOfMiniDoubletsByLayer{Barrel,Endcap} */
  uint32_t lsBarrel[6], lsEndcap[5]; /* getNumberOfSegmentsByLayer{Barrel,Endcap} */
  uint32_t t3Barrel[6], t3Endcap[5]; /* getNumberOfTripletsByLayer{Barrel,Endcap} */
  uint32_t t5Barrel[6], t5Endcap[5]; /* getNumberOfQuintupletsByLayer{Barrel,Endcap} */
  uint32_t reserved[4];
} lst_counts;

/* Static sizes of an event setup. */
typedef struct lst_es_info {
  uint32_t nModules;
  uint32_t nLowerModules;
  uint32_t pixelModule;
  uint32_t nConnectedPixels;
  uint32_t nTotalMDs;      /* MD arena length per event (incl. 100000 pixel MDs) */
  uint32_t nTotalSegments; /* LS arena length per event (incl. 50000 pLS) */
  uint32_t maxTriplets;    /* T3 arena length per event */
  uint32_t maxQuintuplets; /* T5 arena length per event */
  float ptCut;             /* pt cut (GeV) of the module maps: from the geometry directory's
                              "_pt<x>" suffix, 0.8 without one (SDL/Constants.h:102-105) */
} lst_es_info;

/* Last error message of the calling thread (empty if none). */
const char* lst_last_error(void);

/* Launch resources of the library's kernels (registers per thread, the
 * largest block they can be launched with, local and static shared memory). */
int lst_kernel_count(void);
int lst_kernel_attributes(int i, const char** name, int* num_regs, int* max_threads_per_block, size_t* local_bytes,
                          size_t* static_smem_bytes);

/* ------------------------------------------------------------------ ES */
/* Loads the geometry directory (the OT800_IT615_pt0.8 layout: sensor
 * centroids, module connection map, pixel maps, endcap and tilted-barrel
 * orientation) and uploads it to `device`, with the T5 DNN weights from
 * `t5dnn_weights_path` (2337 little-endian float32: w0[38][32], b0[32],
 * w2[32][32], b2[32], w4[32], b4[1]; NULL disables the DNN method).
 * Replaces SDL::loadAndFillESHost + SDL::loadAndFillESDevice
 * (SDL/LSTESData.h:79-80, SDL/LSTESData.cc:79-126). */
int lst_es_load(const char* geometry_dir, const char* t5dnn_weights_path, int device, lst_es** out);
/* lst_es_load with options.  LST_ES_BUILD_ON_DEVICE builds the event setup on
 * `device` from the files' raw records (module re-indexing, detId hash,
 * orientations, partners, module and pixel maps, occupancy caps) instead of
 * on the host; the arrays, and the error messages, are the same.  The host
 * copy of the event setup (lst_es_host_array) is then read back from the
 * device. */
#define LST_ES_BUILD_ON_DEVICE 1u
int lst_es_load_ex(const char* geometry_dir, const char* t5dnn_weights_path, int device, unsigned int flags,
                   lst_es** out);
void lst_es_free(lst_es* es);
/* Loads the geometry on the host only (no device, no upload): for inspecting
 * the event setup.  Such a handle cannot create event sets. */
int lst_es_load_host(const char* geometry_dir, lst_es** out);
/* Host copy of one event-setup array by the reference's name
 * (modules.<field> of SDL/Module.h:161-262, pixelmap.<field> of
 * SDL/PixelMap.h:16-29, endcap.geoMapDetId / endcap.geoMapPhi of
 * SDL/EndcapGeometry.h) or caps.<mdOffset|mdCap|lsOffset|lsCap|t3CapIfUsed|
 * t5CapIfEligible> (the static per-module offsets and occupancy caps). */
int lst_es_host_array(const lst_es* es, const char* name, const void** data, size_t* n_elems, size_t* elem_size);
int lst_es_get_info(const lst_es* es, lst_es_info* out);
/* Sets the T5 DNN working point (the score a candidate must exceed; the
 * reference's is 0.6177366, SDL/Constants.h:145), for every event set on the
 * ES's device. */
int lst_es_set_t5dnn_threshold(lst_es* es, float wp);
/* Replaces the T5 DNN weights (same layout as the file).  The weights live
 * in constant memory of the ES's device and are shared by every event set on
 * that device; call between events. */
int lst_es_set_t5dnn_weights(lst_es* es, const float* weights, size_t n);

/* --------------------------------------------------------------- events */
/* Creates an event set of `n_slots` events holding at most `max_hits` hits
 * each, on the ES's device.  `stream` is a cudaStream_t to run on (NULL: the
 * set creates its own non-blocking stream).  All device memory is allocated
 * here, once.  Replaces the constructor SDL::Event(bool, Queue, ESDeviceData*)
 * (SDL/Event.h:100-111), whose arenas are allocated per event. */
int lst_event_create(lst_es* es, int n_slots, uint32_t max_hits, void* stream, lst_event** out);
void lst_event_destroy(lst_event* ev);
/* Device memory held by the set, in bytes. */
int lst_event_memory(const lst_event* ev, size_t* bytes);
/* Synchronises the set's stream. */
int lst_event_sync(lst_event* ev);
/* The CUDA stream the set runs on (a cudaStream_t). */
void* lst_event_stream(lst_event* ev);
/* Selects the T5 method (default LST_T5_DNN when weights were loaded). */
int lst_event_set_t5_method(lst_event* ev, int method);

/* The quintuplet and pixel stages evaluate their candidates as flat lists and
 * fall back to one warp per module / pLS for events whose candidates overflow
 * the list buffers; the duplicate-removal and cross-cleaning kernels fall back
 * to pair-by-pair tests for events whose objects overflow their shared-memory
 * staging.  on = 1 makes every event take the fallbacks (same results; for
 * testing them). */
int lst_event_set_walk(lst_event* ev, int on);

/* Event::resetEvent (SDL/Event.cc:45): clears slot `slot`'s objects.  Adding
 * hits resets the slot as well. */
int lst_event_reset(lst_event* ev, int slot);

/* Event::addHitToEvent (SDL/Event.cc:151): resets the slot, copies the hits
 * (host or device pointers) and runs the hit preparation and module-range
 * kernels.  Returns LST_STATUS_HIT_CAPACITY (>0) without touching the slot if
 * n > max_hits. */
int lst_event_add_hits(lst_event* ev, int slot, uint32_t n, const float* x, const float* y, const float* z,
                       const uint32_t* detId, const uint32_t* idxInNtuple);

/* Event::addPixelSegmentToEvent (SDL/Event.cc:217; argument order of
 * SDL/Event.h:120-137): copies the pixel line segments and builds their
 * mini-doublets and segment records.  More than 50000 segments are truncated
 * as in the reference (LST_STATUS_PLS_TRUNCATED). */
int lst_event_add_pixel_segments(lst_event* ev, int slot, uint32_t n, const uint32_t* hitIndices0,
                                 const uint32_t* hitIndices1, const uint32_t* hitIndices2,
                                 const uint32_t* hitIndices3, const float* dPhiChange, const float* ptIn,
                                 const float* ptErr, const float* px, const float* py, const float* pz,
                                 const float* eta, const float* etaErr, const float* phi, const int32_t* charge,
                                 const uint32_t* seedIdx, const int32_t* superbin, const int8_t* pixelType,
                                 const int8_t* isQuad);

/* Runs one stage (enum lst_stage) on one slot (the Event::create* members). */
int lst_event_run_stage(lst_event* ev, int slot, int stage);
int lst_event_create_mini_doublets(lst_event* ev, int slot);
int lst_event_create_segments(lst_event* ev, int slot);
int lst_event_create_triplets(lst_event* ev, int slot);
int lst_event_create_quintuplets(lst_event* ev, int slot);
int lst_event_pixel_line_segment_cleaning(lst_event* ev, int slot);
int lst_event_create_pixel_quintuplets(lst_event* ev, int slot);
int lst_event_create_pixel_triplets(lst_event* ev, int slot);
int lst_event_create_track_candidates(lst_event* ev, int slot);

/* Copies the counts of one slot to the host (synchronises the stream).
 * Returns the slot's status bits. */
int lst_event_get_counts(lst_event* ev, int slot, lst_counts* out);

/* Copies one object-store field of a slot to host memory `dst` (synchronises
 * the stream).  `name` is "<store>.<field>" with the reference's store and
 * field names (hits.xs, md.anchorHitIndices, ls.mdIndices, t3.hitIndices,
 * t5.score_rphisum, pt3.hitIndices, pt5.T5Indices, tc.hitIndices,
 * ranges.quintupletModuleIndices, ...).  The full array (its arena length)
 * is described by *n_elems and *elem_size; min(n_elems, capacity) elements
 * are copied.  dst may be NULL to query the length.  Replaces the getters
 * getHits() ... getTrackCandidates() (SDL/Event.cc:1489-1805). */
int lst_event_get_field(lst_event* ev, int slot, const char* name, void* dst, size_t capacity, size_t* n_elems,
                        size_t* elem_size);
/* Device address of a field of a slot (for zero-copy consumers). */
int lst_event_field_device_ptr(lst_event* ev, int slot, const char* name, void** dptr, size_t* n_elems,
                               size_t* elem_size);
/* Number of fields, the i-th name, and its element type: *elem_size bytes of
 * kind 'f' (IEEE float), 'i' (signed integer) or 'u' (unsigned integer). */
int lst_field_count(void);
const char* lst_field_name(int i);
int lst_field_info(int i, const char** name, size_t* elem_size, char* kind);

/* --------------------------------------------------------------- batches */
/* Packed per-event input, one contiguous little-endian blob per event:
 *   uint32 nHits, uint32 nPLS, uint32 reserved[2],
 *   float x[nHits], y[nHits], z[nHits], uint32 detId[nHits], idxInNtuple[nHits],
 *   uint32 hitIndices0..3[nPLS], float dPhiChange, ptIn, ptErr, px, py, pz, eta,
 *   etaErr, phi [nPLS each], int32 charge[nPLS], uint32 seedIdx[nPLS],
 *   int32 superbin[nPLS], int8 pixelType[nPLS], int8 isQuad[nPLS]
 * (lst_packed_size gives the byte size).  `blob_offsets[i]` is the byte
 * offset of event i's blob inside `blobs`; each offset is a multiple of 16.
 * lst_batch_upload copies `total_bytes` of host (preferably pinned) memory in
 * one transfer and unpacks events into slots [first, first + count), i.e. it
 * performs addHitToEvent + addPixelSegmentToEvent for all of them. */
size_t lst_packed_size(uint32_t n_hits, uint32_t n_pls);
int lst_batch_upload(lst_event* ev, int first, int count, const void* blobs, size_t total_bytes,
                     const uint64_t* blob_offsets);
/* Repeats the unpacking of the last uploaded inputs of slots [first,
 * first + count) (as lst_batch_upload or lst_batch_upload_seeds without the
 * host-to-device copy), for re-running events whose inputs are already
 * resident on the device.  The slots must lie inside the last upload. */
int lst_batch_ingest(lst_event* ev, int first, int count);
/* Input staging that overlaps the next batch's host-to-device copy with the
 * current batch's stages (no reference counterpart).  lst_batch_stage starts
 * the copy of packed events (the lst_batch_upload layout, or with
 * seed_layout = 1 the lst_batch_upload_seeds one) into one of two device
 * staging buffers on the set's own copy stream and returns at once; blobs
 * must be pinned host memory (pageable memory is copied synchronously) and
 * must stay unchanged until the copy has run.  lst_batch_ingest_staged makes
 * the set's stream wait for that copy and ingests the staged events into
 * their slots, as lst_batch_upload does after its copy.  One batch can be
 * staged at a time; staging the next one while the current one runs its
 * stages (and before reading its output) hides the copy. */
int lst_batch_stage(lst_event* ev, int first, int count, const void* blobs, size_t total_bytes,
                    const uint64_t* blob_offsets, int seed_layout);
int lst_batch_ingest_staged(lst_event* ev);
/* Runs stages [first_stage, last_stage] for slots [first, first + count). */
int lst_batch_run(lst_event* ev, int first, int count, int first_stage, int last_stage);
/* As lst_batch_run, replayed from a CUDA graph: the first call for a given
 * (first, count, stage range, T5 method) captures the launches on the set's
 * stream into a graph and every later call replays it with one launch.  The
 * first call must not run while another capture is active on the stream. */
int lst_batch_run_graph(lst_event* ev, int first, int count, int first_stage, int last_stage);
/* Copies the counts of slots [first, first + count) into out[count]. */
int lst_batch_get_counts(lst_event* ev, int first, int count, lst_counts* out);

/* ---------------------------------------------- CMSSW inputs (LST::run) */
/* The inputs of LST::run / LST::prepareInput (SDL/LST.h:32-52,
 * SDL/LST.cc:12-32,175-194): per pixel seed its momentum at the point of
 * closest approach (see_px/py/pz), impact parameters (see_dxy, see_dz),
 * errors (see_ptErr, see_etaErr), position and momentum at its last hit
 * (see_stateTrajGlb*), charge (see_q) and pixel-hit indices; the outer-tracker
 * hits as ph2_detId/x/y/z.  see_hitIdx, a vector<vector<int>> in the
 * reference, is flattened: seed i's indices are see_hitIdx[see_hitIdx_offsets[i]
 * .. see_hitIdx_offsets[i + 1]) with see_hitIdx_offsets[0] = 0 (n_seeds + 1
 * entries).  Kept seeds need at least three indices (the reference reads three
 * of every kept seed); a kept seed with fewer is dropped and the slot gets
 * LST_STATUS_INVALID_INPUT. */
typedef struct lst_seed_input {
  uint32_t n_seeds;
  const float* see_px;
  const float* see_py;
  const float* see_pz;
  const float* see_dxy;
  const float* see_dz;
  const float* see_ptErr;
  const float* see_etaErr;
  const float* see_stateTrajGlbX;
  const float* see_stateTrajGlbY;
  const float* see_stateTrajGlbZ;
  const float* see_stateTrajGlbPx;
  const float* see_stateTrajGlbPy;
  const float* see_stateTrajGlbPz;
  const int32_t* see_q;
  const uint32_t* see_hitIdx_offsets;
  const int32_t* see_hitIdx;
  uint32_t n_ph2;
  const uint32_t* ph2_detId;
  const float* ph2_x;
  const float* ph2_y;
  const float* ph2_z;
} lst_seed_input;

/* Packed form of one event's lst_seed_input for lst_batch_upload_seeds:
 * lst_seed_packed_size bytes (a multiple of 16); lst_seed_pack writes it into
 * host memory `dst` of `capacity` bytes (-1 if it does not fit or an array is
 * missing; the offsets are checked to ascend). */
size_t lst_seed_packed_size(uint32_t n_ph2, uint32_t n_seeds, uint32_t n_seed_hits);
int lst_seed_pack(const lst_seed_input* in, void* dst, size_t capacity);
/* As lst_batch_upload for packed seed events: one host-to-device copy, then
 * on the device the seed conversion of LST::prepareInput (SDL/LST.cc:175-365,
 * including its phi(r3LH - p3LH) "deltaPhi" of :265) followed by
 * addHitToEvent + addPixelSegmentToEvent, for slots [first, first + count). */
int lst_batch_upload_seeds(lst_event* ev, int first, int count, const void* blobs, size_t total_bytes,
                           const uint64_t* blob_offsets);
/* LST::prepareInput + addHitToEvent + addPixelSegmentToEvent for one slot
 * (SDL/LST.cc:33-72): the outer-tracker hits, then per kept seed (pT above
 * 0.8 - 2 ptErr) three or four pseudo-hits and one pixel line segment. */
int lst_event_prepare_input(lst_event* ev, int slot, const lst_seed_input* in);

/* Track-candidate output of LST::getOutput (SDL/LST.cc:367-427) for slots
 * [first, first + count), flattened over the events: candidate k of the batch
 * has type[k], seedIdx[k] (pixelSeedIndex) and len[k] input-ntuple hit
 * indices, stored back to back in hits[].  Event i owns candidates
 * [event_tc_offsets[i], event_tc_offsets[i + 1]) and hits
 * [event_hit_offsets[i], event_hit_offsets[i + 1]); both offset arrays hold
 * count + 1 entries and are always filled.  If tc_capacity or hits_capacity
 * is too small, nothing else is written and the call returns -1. */
typedef struct lst_output {
  uint32_t* hits;
  size_t hits_capacity;
  uint32_t* len;
  int32_t* seedIdx;
  int16_t* type;
  size_t tc_capacity;
  uint64_t* event_tc_offsets;
  uint64_t* event_hit_offsets;
} lst_output;
int lst_batch_get_output(lst_event* ev, int first, int count, lst_output* out);

/* LST::run (SDL/LST.cc:12-161) on one slot: lst_event_prepare_input, all
 * eight stages, then, if `out` is not NULL, the output accessors hits(),
 * len(), seedIdx(), trackCandidateType() (SDL/LST.h:53-56) as
 * lst_batch_get_output with count = 1.  The slot keeps its objects until it
 * is reset or refilled (the reference discards its Event at the end of run). */
int lst_run(lst_event* ev, int slot, const lst_seed_input* in, lst_output* out);

/* lst_batch_get_output without any device allocation (no reference
 * counterpart: the reference allocates its host copies in getOutput).
 * lst_batch_get_output grows its device staging buffer with cudaMalloc when a
 * batch needs more room; callers that cannot allocate device memory at that
 * point -- a framework whose caching allocator owns the device memory budget,
 * or a producer that must not stall other streams with the device-wide
 * synchronisation of cudaMalloc / cudaFree -- call this one.  It stages in a
 * fixed 4 MiB device array compiled into the library (about 20 PU200-shaped
 * events per call) and rejects a call whose output does not fit (or of more
 * than 1023 events) with an error naming the size: split the slot range.  The
 * first call on each device looks the array up (cudaGetSymbolAddress with
 * that device current); make that first call before any stream capture.  The
 * looked-up address is kept while an event setup (lst_es) is alive on the
 * device and forgotten when the last one is freed; a cudaDeviceReset while one
 * is alive invalidates it together with its event sets.  All
 * event sets of a device share the array, so calls that overlap in time (on
 * different streams or host threads) race: serialise them. */
int lst_batch_get_output_static(lst_event* ev, int first, int count, lst_output* out);

/* ---------------------------------------------------------- accounting */
/* Number of kernels the set has launched since it was created. */
int lst_event_launches(const lst_event* ev, uint64_t* n);
/* With profiling on, every launch of the set is bracketed by CUDA events on
 * its stream; lst_event_get_profile synchronises, sums the elapsed times per
 * kernel since profiling was switched on (or last read) and clears them. */
typedef struct lst_kernel_time {
  const char* name;
  uint64_t launches;
  double total_ms;
} lst_kernel_time;
int lst_event_set_profiling(lst_event* ev, int on);
int lst_event_get_profile(lst_event* ev, lst_kernel_time* out, int capacity, int* n_kernels);

/* ---------------------------------------------------------- autotuner */
/* No reference counterpart (the reference launches with fixed work
 * divisions, SDL/Event.cc).  The kernels that do most of the work take their
 * launch shape from the event set: warps per block and resident blocks per
 * SM across the batch (each event gets blocks_per_sm x SMs / events blocks).
 * Object lists do not depend on the shape. */
int lst_tune_kernel_count(void);
const char* lst_tune_kernel_name(int k);
int lst_event_set_launch_shape(lst_event* ev, int k, int warps_per_block, int blocks_per_sm);
int lst_event_get_launch_shape(const lst_event* ev, int k, int* warps_per_block, int* blocks_per_sm);
/* Hash of the loaded geometry (module map, connections, static arenas). */
uint64_t lst_es_geometry_hash(const lst_es* es);
/* Times a sweep of launch shapes (1-8 warps per block x 16-128 blocks per SM)
 * on slots [first, first + count), whose inputs must be resident from the
 * last upload, keeps the fastest shape per kernel, and checks that every
 * shape gave the same object counts.  With a cache path the result is stored
 * there under a key of geometry hash, device name, batch size and library
 * build, replacing an older entry of that key; lst_autotune_load applies the
 * stored entry (1 if found, 0 if not). */
int lst_autotune(lst_event* ev, int first, int count, const char* cache_path);
int lst_autotune_load(lst_event* ev, int count, const char* cache_path);

/* ---------------------------------------------------------- T5 classifier */
/* Classifier-stage probe (no reference counterpart; it serves retraining the
 * T5 DNN of SDL/NeuralNetwork.h): after createQuintuplets, every quintuplet
 * candidate of slots [first, first + count) that passes all cuts before the
 * DNN decision is appended to the DEVICE buffers given: its 38 DNN inputs
 * (feat, capacity x 38, in the order of SDL/NeuralNetwork.h:74-114), the
 * loaded weights' score, the cut-only method's decision, the rz-fit tight
 * flag, its 10 hit indices (event-local) and its slot.  *n_found receives the
 * number of candidates found (entries beyond capacity are dropped). */
int lst_batch_t5_probe(lst_event* ev, int first, int count, float* feat, float* score, uint8_t* cut_pass,
                       uint8_t* rz_tight, uint32_t* hits, int32_t* event_index, uint32_t capacity,
                       uint32_t* n_found);

/* Forward and backward passes of the T5 DNN (38 -> 32 ReLU -> 32 ReLU -> 1)
 * for training, on device buffers in the caller's stream (a cudaStream_t).
 * weights: 2337 floats in the weight-file layout.  Forward: x (n x 38) ->
 * h1, h2 (n x 32, kept for the backward pass), logit (n).  Backward: from
 * dlogit (n, the loss gradient w.r.t. the logits) -> grad (2337, same layout
 * as the weights); scratch needs lst_t5dnn_scratch_floats(n) floats.  The
 * reductions run in a fixed order, so the gradient is deterministic. */
int lst_t5dnn_forward(const float* weights, const float* x, int n, float* h1, float* h2, float* logit, void* stream);
size_t lst_t5dnn_scratch_floats(int n);
int lst_t5dnn_backward(const float* weights, const float* x, const float* h1, const float* h2, const float* dlogit,
                       int n, float* grad, float* scratch, void* stream);
/* Last error message of the two training entry points above. */
const char* lst_t5dnn_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* LST_B200_H */
