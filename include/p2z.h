/*
 * p2z.h -- C ABI of the B200 propagate-to-z + Kalman-update library (libp2z.so).
 *
 * The reference benchmark has no library boundary: its "API" is a set of C++
 * free functions compiled into each executable together with main().  This
 * header is the thin extern "C" layer that replaces them.  Every entry point
 * names the reference interface it stands in for (file:line inside the
 * reference project).  Signatures use plain pointers, sizes and enums only.
 *
 * Data layout (unchanged from the reference, src/propagate-toz-test_OMP.cpp:57-125):
 *   A track batch (MPTRK) of width B holds element p of track t at data[t + p*B]:
 *     float par[6*B]   x, y, z, ipt (= 1/pT), phi, theta
 *     float cov[21*B]  packed lower triangle of the symmetric 6x6 covariance,
 *                      (i,j) with i >= j at i*(i+1)/2 + j   (SymOffsets66, :52-55)
 *     int   q[B]       charge
 *   sizeof(MPTRK) = 28*B*4 bytes.
 *   A hit batch (MPHIT) of width B:
 *     float pos[3*B]   x, y, z
 *     float cov[6*B]   packed lower triangle of the 3x3 hit covariance
 *   sizeof(MPHIT) = 9*B*4 bytes.
 *   Track batches of event e are consecutive (bTk: batch ib of event e at ib + nb*e,
 *   :147-153).  The hits of track batch b on layer l are hit batch l + nlayer*b
 *   (bHit, :215-217), i.e. the layers of a batch are contiguous.
 *
 * Uneven events (no counterpart in the reference, which fixes ntrks per event):
 *   event e holds ceil(n_e/B) batches; the batches of all events are consecutive
 *   and the last batch of an event may be partly filled.  A per-track-slot hit
 *   mask (one uint32 per slot, slot = batch*B + t, bit l = "track has a hit on
 *   layer l") marks missing layers; a layer whose bit is clear is skipped
 *   entirely (neither propagated to nor updated with).  Padding slots carry
 *   mask 0 and are copied through unchanged.
 *
 * SoA layout (p2z_config.layout = P2Z_LAYOUT_SOA; no counterpart in the
 * reference): the same slots (slot = batch*B + t, events padded to multiples of
 * bsize as above) stored as one batch spanning all nslots = nbatches*bsize
 * slots: tracks as float[28][nslots] (element p of slot s at p*nslots + s) and
 * hits as float[nlayer][9][nslots] (element p of layer l at
 * (l*9 + p)*nslots + s).  Masks are indexed by slot in both layouts.
 *
 * Threading: a p2z_context belongs to one host thread at a time.  Device-side
 * work is ordered on the stream passed in (or the context's own stream).
 */
#ifndef P2Z_H
#define P2Z_H

/* The reference's sources define their sizes as macros (bsize, nevts, ntrks,
 * nlayer, nb, NITER, nthreads, smear, N: src/propagate-toz-test_OMP.cpp:18-41,
 * :295) before any code.  They are set aside while this header compiles and
 * restored at its end, so it can be included before or after them.  In code
 * that sees those macros, fill a p2z_config with p2z_config_init: a member
 * access such as cfg.bsize would expand the macro. */
#pragma push_macro("bsize")
#undef bsize
#pragma push_macro("nevts")
#undef nevts
#pragma push_macro("ntrks")
#undef ntrks
#pragma push_macro("nlayer")
#undef nlayer
#pragma push_macro("nb")
#undef nb
#pragma push_macro("NITER")
#undef NITER
#pragma push_macro("nthreads")
#undef nthreads
#pragma push_macro("smear")
#undef smear
#pragma push_macro("N")
#undef N

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define P2Z_ABI_VERSION 2

/* Field constant of the reference's OMP/TBB/CUDA_v4 family:
 * kfact = 100/(-0.299792458*3.8112) (src/propagate-toz-test_OMP.cpp:622),
 * the 3.8 T solenoid.  p2z_config.kfact = 0 selects it. */
#define P2Z_KFACT_DEFAULT (-87.5220642f)

typedef enum p2z_status {
  P2Z_OK = 0,
  P2Z_BAD_ARG = 1,           /* invalid size, pointer or enum value */
  P2Z_OOM = 2,               /* device or pinned-host allocation failed / budget exceeded */
  P2Z_NONFINITE_INPUT = 3,   /* P2Z_FLAG_CHECK_INPUTS found a NaN/Inf in the inputs */
  P2Z_SINGULAR = 4,          /* P2Z_FLAG_STRICT: a residual covariance had det <= 0 */
  P2Z_TIMEOUT = 5,           /* a bounded wait ran out (serving, or a staged kernel's copy wait) */
  P2Z_CUDA_ERROR = 6,        /* a CUDA runtime call failed; see p2z_last_error() */
  P2Z_NO_DEVICE = 7,         /* no usable CUDA device */
  P2Z_UNSUPPORTED = 8,       /* valid but not built (e.g. an unsupported bsize) */
  P2Z_NOT_READY = 9          /* serving: the request has not completed yet */
} p2z_status;

/* Measurement-update flavours.
 *  V2            the reference's KalmanUpdate_v2 (src/propagate-toz-test_OMP.cpp:503-620): 2-D (x,y)
 *                update, evaluated in FP32 with no FP64 instruction -- Kahan's compensated 2x2
 *                determinant and a Newton-refined reciprocal, positions anchored at the last hit, and
 *                each track's first update in the Joseph form (I-KH)C(I-KH)^T + KVK^T (later
 *                updates: the reference's C - K H C).  With P2Z_FLAG_REFERENCE_ROUNDING: the
 *                reference's own FP32 expressions instead, its determinant in FP64.
 *  V2_COMP       the same estimator and evaluation with float-pair (double-float) accumulators for
 *                x and y instead of anchored positions; no FP64 either.
 *  3X3_F64       3-D (x,y,z) update; the 3x3 residual covariance H C H^T + V is inverted and the
 *                covariance is updated in the Joseph form (I-KH)C(I-KH)^T + KVK^T, both in FP64.
 *                Basis: the reference's 3x3 KalmanUpdate (v1, :375-501), off its active path.
 *  3X3_COMP      the 3-D Joseph update in FP32 only, with compensated cofactors/determinant.
 *  F64           everything (propagation and V2 update) in FP64 on the GPU, for precision studies. */
typedef enum p2z_update_kind {
  P2Z_UPDATE_V2 = 0,
  P2Z_UPDATE_V2_COMP = 1,
  P2Z_UPDATE_3X3_F64 = 2,
  P2Z_UPDATE_3X3_COMP = 3,
  P2Z_UPDATE_F64 = 4
} p2z_update_kind;

/* How the work is laid onto the GPU.
 *  AUTO        FLAT for uniform events, PERSISTENT when event_ntrks or a hit mask is given.
 *  FLAT        one launch over every track slot of every event.
 *  PER_EVENT   one launch per event (the reference's launch-per-chunk form,
 *              src/propagate-toz-test_CUDA_v4.cu:970-986, taken down to one event per launch).
 *  PERSISTENT  one persistent launch (grid = resident CTAs) whose warps take
 *              work items of 32 slots (16 with two threads per track) from a
 *              device queue; replayed as a CUDA graph.
 *  STAGED      the persistent form with each warp's hit tiles streamed through
 *              shared memory by bulk asynchronous copies, several layers ahead,
 *              and the next batch's tracks copied in during the current one.
 *              bsize 32, AOSOA layout and 16-byte aligned track and hit arrays
 *              only (P2Z_UNSUPPORTED otherwise).  p2z_run runs its chunks flat. */
typedef enum p2z_schedule {
  P2Z_SCHED_AUTO = 0,
  P2Z_SCHED_FLAT = 1,
  P2Z_SCHED_PER_EVENT = 2,
  P2Z_SCHED_PERSISTENT = 3,
  P2Z_SCHED_STAGED = 4
} p2z_schedule;

/* Array layouts (see the top of this file). */
typedef enum p2z_layout {
  P2Z_LAYOUT_AOSOA = 0, /* the reference's MPTRK / MPHIT batches */
  P2Z_LAYOUT_SOA = 1    /* one array per element over all slots */
} p2z_layout;

/* Flags */
#define P2Z_FLAG_CHECK_INPUTS 0x1u  /* scan the input words the pass reads for NaN/Inf ->
                                       P2Z_NONFINITE_INPUT: the 27 floating-point track words of
                                       every slot with a present layer and, on each present layer,
                                       the hit words the update kind reads (6 for the 2-D updates,
                                       9 for the 3-D ones); padding slots and absent layers are not
                                       read and not scanned.  p2z_run_device: before the pass,
                                       synchronously, and the pass does not run; p2z_run: each
                                       chunk after its copy, the pass still runs */
#define P2Z_FLAG_STRICT       0x2u  /* return P2Z_SINGULAR if any det <= 0 was met */
#define P2Z_FLAG_NO_GRAPH     0x4u  /* PERSISTENT, and p2z_run with page-locked buffers: enqueue
                                       directly instead of replaying a recorded graph */
#define P2Z_FLAG_ACCURATE_TRIG 0x8u /* sin and 1 - cos of every per-layer angle from sincosf of its
                                       half (default: Taylor polynomials for the helix angle alpha
                                       when |alpha| <= 0.5, for cosP*sin(alpha) and for the phi
                                       offset from its anchor; sincosf beyond 0.5 rad) */
#define P2Z_FLAG_FULL_HITS    0x10u /* p2z_run: copy all 9 hit words per track even for the 2-D
                                       updates (default: only the 6 words they read) */
#define P2Z_FLAG_PER_EVENT_STREAMS 0x40u /* PER_EVENT: issue the per-event launches round-robin on 10
                                       streams forked from the run's stream and joined back to it, as
                                       the reference's GPU build spreads its launches over num_streams
                                       = 10 (src/propagate-toz-test_CUDA_v4.cu:40-41, :972-986); the
                                       default issues them in order on the run's stream */
#define P2Z_FLAG_SORT_WINDOWS 0x80u /* masked runs, FLAT / PERSISTENT: process each window of 128
                                       consecutive slots in order of the slots' hit counts (a 1-byte
                                       permutation the run computes on the device), so a warp's 32
                                       tracks take similar numbers of steps.  Per-track results are
                                       the same.  On the uneven benchmark sample lane utilisation
                                       rises from 60% to 85% and the persistent pass is 13% faster;
                                       a warp's loads then reach 4 batches, so on even work (every
                                       mask alike) it only costs.  p2z_autotune measures both for
                                       masked runs, and runs with schedule AUTO sort when that
                                       measured faster.  Packing an event's tracks in order of hit
                                       count (p2z_pack_by_hits_device, or when the arrays are built)
                                       gains more (99%) */
#define P2Z_FLAG_REFERENCE_ROUNDING 0x20u /* P2Z_UPDATE_V2 only: evaluate the reference's own FP32
                                       expressions, type promotions and operation order, every
                                       operation separately rounded, with correctly rounded
                                       sin/cos -- the reference's results bit for bit where its
                                       C library's sinf/cosf are correctly rounded.  Default: the
                                       precise evaluation (versine form, positions anchored
                                       at the last hit, direction anchored and advanced by
                                       summed angle offsets, all FP32), within 5e-6 of an FP64
                                       evaluation. */

typedef struct p2z_config {
  int32_t abi_version;   /* must be P2Z_ABI_VERSION */
  int32_t bsize;         /* AOSOA batch width B: 8, 16, 32 or 64 (reference macro bsize, :22-24) */
  int64_t nevts;         /* number of events (reference macro nevts, :18-20) */
  int64_t ntrks;         /* tracks per event, uniform form: a multiple of bsize
                            (reference macro ntrks, nb = ntrks/bsize, :25-29); ignored
                            when event_ntrks is given */
  int32_t nlayer;        /* layers, 1..32 (reference macro nlayer, :35-37) */
  int32_t niter;         /* passes over the whole input (reference NITER, :31-33); each pass
                            recomputes the outputs from the inputs; 0 is treated as 1,
                            negative is P2Z_BAD_ARG */
  float kfact;           /* 0 -> P2Z_KFACT_DEFAULT; not finite -> P2Z_BAD_ARG */
  int32_t update;        /* p2z_update_kind */
  int32_t schedule;      /* p2z_schedule; AUTO -> the schedule p2z_autotune measured best on
                            this context for the same key, else the rule under p2z_schedule */
  int32_t block_threads; /* threads per CTA, a multiple of 32 in 32..256; 0 -> the value
                            p2z_autotune measured best on this context for the same update,
                            flags, bsize, layout and masking, else 128 */
  uint32_t flags;        /* P2Z_FLAG_*; any other bit is P2Z_BAD_ARG */
  int32_t layout;        /* p2z_layout of the track, hit and output arrays */
  /* Uneven form (optional, host memory): nevts track counts.  NULL -> uniform. */
  const int64_t *event_ntrks;
  int32_t threads_per_track; /* 1, or 2 (P2Z_UPDATE_V2 without REFERENCE_ROUNDING; FLAT,
                            PER_EVENT and PERSISTENT schedules): lanes 2i and 2i+1 of a warp
                            hold the same track and split the propagation of its covariance,
                            with bit-identical results.  0 -> the value p2z_autotune measured
                            best on this context for the same update, flags, bsize, layout
                            and masking, else 1.  No counterpart in the reference (one thread
                            per track in every GPU version, src/propagate-toz-test_CUDA_v4.cu:
                            761-775) */
} p2z_config;

/* Fills *cfg for the uniform form: abi_version, the sizes given, one pass,
 * P2Z_UPDATE_V2, and every other field 0 (P2Z_SCHED_AUTO, block size and
 * threads per track from the autotuner or their defaults, no flags, AOSOA,
 * P2Z_KFACT_DEFAULT, no event_ntrks).  Callers whose code defines the
 * reference's size macros pass them here
 * (p2z_config_init(&cfg, bsize, nevts, ntrks, nlayer)) instead of writing
 * cfg.bsize = bsize, which the macros would expand.  Checks nothing but cfg:
 * the run entry points validate the config. */
p2z_status p2z_config_init(p2z_config *cfg, int32_t bsize, int64_t nevts, int64_t ntrks, int32_t nlayer);

/* Filled by the run entry points (optional out-parameter). */
typedef struct p2z_stats {
  double kernel_ms;        /* device time of the hot-path launches (CUDA events), all iterations */
  double h2d_ms;           /* host->device copy time (p2z_run only) */
  double d2h_ms;           /* device->host copy time (p2z_run only) */
  double total_ms;         /* device time from first copy to last copy */
  int64_t track_slots;     /* slots processed per iteration (batches * bsize) */
  int64_t updates;         /* track-layer updates performed per iteration (present hits) */
  int64_t h2d_bytes;
  int64_t d2h_bytes;
  int32_t launches;        /* hot-path kernel launches, all iterations */
  int32_t singular;        /* 1 if a residual covariance with det <= 0 was met */
} p2z_stats;

typedef struct p2z_context p2z_context;

/* ---- context -------------------------------------------------------------- */

/* Create a context on CUDA device `device` (the current device when < 0).
 * No counterpart in the reference (its main owns its device buffers directly,
 * src/propagate-toz-test_CUDA_v4.cu:921-947). */
p2z_status p2z_create(int device, p2z_context **out);
p2z_status p2z_destroy(p2z_context *ctx);
const char *p2z_status_string(p2z_status s);
/* Last detailed error message of this context ("" if none); ctx may be NULL for
 * the most recent context-free failure. */
const char *p2z_last_error(const p2z_context *ctx);
/* Library/ABI identification: returns P2Z_ABI_VERSION, fills a build string. */
int p2z_version(char *buf, size_t buflen);

/* ---- sizes ---------------------------------------------------------------- */

/* Number of track batches described by cfg (uniform: nevts*ntrks/bsize; uneven:
 * sum over events of ceil(n_e/bsize)); -1 on a bad config. */
int64_t p2z_num_batches(const p2z_config *cfg);
size_t p2z_sizeof_mptrk(int bsize);   /* 28*bsize*4 */
size_t p2z_sizeof_mphit(int bsize);   /* 9*bsize*4 */

/* ---- the hot path --------------------------------------------------------- */

/* Full pass from HOST memory: copies tracks and hits to the device, runs
 * propagateToZ + KalmanUpdate for every present layer of every track, copies
 * the updated tracks back.  Replaces the reference's timed region in its
 * include_data mode (src/propagate-toz-test_CUDA_v4.cu:966-990) and the CPU
 * hot loop (src/propagate-toz-test_OMP.cpp:731-748).
 *   trk_in   MPTRK[nbatches]            (host)
 *   hits     MPHIT[nlayer*nbatches]     (host)
 *   hit_mask uint32[nbatches*bsize]     (host, optional, see above)
 *   trk_out  MPTRK[nbatches]            (host; may equal trk_in)
 * Host buffers that are page-locked (cudaHostAlloc / p2z_host_alloc) are
 * copied asynchronously; pageable ones go through a staging path.  The work is
 * split into up to 16 chunks whose copies and passes alternate between two
 * streams.  With page-locked buffers (all of trk_in, hits, trk_out and
 * hit_mask when given) and a pipeline of 4 or more chunk passes (256 or more
 * batches; chunks x niter) or per-event launches (events x niter), the whole
 * pipeline is recorded as a CUDA graph on the first call and replayed by later
 * calls with the same config, host buffers and internal device buffers, so
 * that a call costs one graph launch; a call that differs in any of them
 * records again.  Shorter pipelines are enqueued directly, which lets their
 * first copy start while the rest is enqueued.  P2Z_FLAG_NO_GRAPH enqueues
 * every copy and kernel directly.  Synchronous: returns when trk_out holds
 * the results. */
p2z_status p2z_run(p2z_context *ctx, const p2z_config *cfg, const void *trk_in, const void *hits,
                   const uint32_t *hit_mask, void *trk_out, p2z_stats *stats);

/* Same pass on DEVICE-resident buffers, enqueued on `stream` (a cudaStream_t;
 * NULL = the context's stream, cudaStreamLegacy = the legacy default stream).
 * The context's stream is not ordered with any other: a caller whose buffers
 * come from work on another stream passes that stream, or synchronises it
 * first.  Returns after enqueueing (asynchronous) unless stats != NULL (it
 * then synchronises to fill the timings), P2Z_FLAG_STRICT is set (it
 * synchronises to read the status: P2Z_SINGULAR, or P2Z_TIMEOUT from a staged
 * wait) or P2Z_FLAG_CHECK_INPUTS is set (the scan before the pass).  The PERSISTENT schedule's
 * graph is recorded on the context's stream and replayed on `stream`; while
 * `stream` is itself being captured, the kernels are launched into it directly.
 * d_trk_out must not alias d_trk_in.  Calls on one context whose work
 * overlaps on the GPU (different streams, as the reference's GPU build issues
 * its chunks) share the context's device scratch: with the FLAT schedule
 * (the rule for runs without masks) and the default flags they share only the
 * status word, whose bits the kernels only set, and may overlap; with the
 * PERSISTENT or STAGED schedule (work counter), P2Z_FLAG_SORT_WINDOWS (window
 * permutation), uneven events given without a mask (padding mask), stats or
 * P2Z_FLAG_CHECK_INPUTS (status reset) they must not: order those streams, or
 * use one context per stream.  Replaces GPUsequence/GPUsequenceR
 * (src/propagate-toz-test_CUDA_v4.cu:746-828). */
p2z_status p2z_run_device(p2z_context *ctx, const p2z_config *cfg, const void *d_trk_in, const void *d_hits,
                          const uint32_t *d_hit_mask, void *d_trk_out, void *stream, p2z_stats *stats);

/* One layer step on device buffers, in place on d_trk (nbatches MPTRK of width
 * bsize): what = 1 propagateToZ (src/propagate-toz-test_OMP.cpp:623-682),
 * 2 KalmanUpdate_v2 (:503-620), 3 both.  `update` must be P2Z_UPDATE_V2 (any
 * other kind returns P2Z_UNSUPPORTED: the step form exists for the
 * reference's own layer loop).  The reference's FP32 expressions with every
 * operation rounded separately (the P2Z_FLAG_REFERENCE_ROUNDING arithmetic),
 * the full 21-element covariance (its z row may be non-zero); kfact 0 ->
 * P2Z_KFACT_DEFAULT.  The hits used are those of `layer` in the standard hit
 * array of nlayer layers.  Runs on the context's stream; synchronous. */
p2z_status p2z_step_device(p2z_context *ctx, int bsize, int64_t nbatches, void *d_trk, const void *d_hits,
                           int nlayer, int layer, int what, int update, float kfact);

/* The same pass as p2z_run_device with the persistent schedule, for callers
 * that cannot allocate device memory: applications whose device memory belongs
 * to another allocator that must account for every byte (a framework's caching
 * allocator, an experiment's memory manager with fixed budgets), and
 * latency-critical paths on which cudaMalloc/cudaFree are not allowed because
 * they can synchronise the whole device.  No counterpart in the reference.
 * It needs no p2z_context (creating one allocates) and calls no allocating
 * routine: its scratch -- the work counter, the status word and, for uneven
 * events given without a hit mask, the padding mask and event offsets -- is a
 * fixed array of about 5 MB inside the library, which every GPU that loads the
 * library holds until the process exits.  Limits: an uneven run without a hit
 * mask may have at most P2Z_NOALLOC_MAX_SLOTS track slots and
 * P2Z_NOALLOC_MAX_EVENTS events (larger runs return P2Z_BAD_ARG with a message
 * in p2z_last_error(NULL)); uniform runs and runs with a caller-provided mask
 * have no size limit.  AOSOA layout only (P2Z_UNSUPPORTED otherwise).  The
 * schedule, block size 0, threads_per_track and the P2Z_FLAG_SORT_WINDOWS /
 * _PER_EVENT_STREAMS flags do not apply (always the persistent pass in stored
 * slot order, one thread per track, 128 threads per CTA unless block_threads
 * is set); niter passes are run.  No
 * status comes back from the device, so P2Z_FLAG_STRICT and
 * P2Z_FLAG_CHECK_INPUTS return P2Z_UNSUPPORTED.  For uneven events without a
 * mask, event_ntrks is read from host memory when the call is made.
 * Enqueued on `stream` (a cudaStream_t; NULL is the legacy default stream:
 * there is no context stream here) on the current device; returns after
 * enqueueing.  The first call on a device looks up the scratch array's device
 * address (once per device, with that device current) and keeps it for the
 * life of the process, so a device that is reset (cudaDeviceReset) must not
 * be used with this entry point afterwards in that process.  All calls share
 * the one scratch array and each call resets what must start at zero, so
 * calls whose work overlaps on the GPU (different streams, or concurrent host
 * threads) race on it: serialise them. */
#define P2Z_NOALLOC_MAX_SLOTS (1 << 20)
#define P2Z_NOALLOC_MAX_EVENTS (1 << 16)
p2z_status p2z_run_device_noalloc(const p2z_config *cfg, const void *d_trk_in, const void *d_hits,
                                  const uint32_t *d_hit_mask, void *d_trk_out, void *stream);

/* ---- layouts and tuning (no counterpart in the reference) ------------------ */

/* Copy tracks, hits and (optionally) masks of the same events from the layout
 * and bsize `from` describes to those `to` describes, on the device, enqueued
 * on `stream` (NULL = the context's stream).  from and to must describe the
 * same events: equal nevts and nlayer and the same track count per event
 * (uniform ntrks or event_ntrks).  Padding slots of the destination get zero
 * tracks and hits and, when masks are converted, mask 0.  Pass both masks or
 * neither.  Destination buffers must not overlap the sources. */
p2z_status p2z_relayout_device(p2z_context *ctx, const p2z_config *from, const p2z_config *to,
                               const void *d_trk_in, const void *d_hits_in, const uint32_t *d_mask_in,
                               void *d_trk_out, void *d_hits_out, uint32_t *d_mask_out, void *stream);

/* Packing tracks with missing layers in order of hit count.  A warp's 32
 * tracks take as many steps as the one with the most hits, so an uneven
 * sample runs fastest when each batch holds tracks of similar hit counts.
 * p2z_pack_by_hits_device writes a copy of cfg's AOSOA arrays (tracks, hits
 * and, when given, masks) in which every event's tracks are in order of
 * decreasing hit count -- a stable order: equal counts keep their order; every
 * event keeps its own slots and its padding last -- and the permutation in
 * d_perm, 2 * nbatches * bsize int64: d_perm[s] = the input slot that packed
 * slot s holds, and after those the inverse, d_perm[nslots + q] = the packed
 * slot of input slot q.
 * Runs on the packed arrays give each track the bits it gets in the caller's
 * order; p2z_unpack_tracks_device writes a packed output back in the caller's
 * order.  No mask: every track has every layer and the order is unchanged.
 * The copies must not alias the inputs.  Pack: synchronous (its scratch, about
 * 32 bytes a slot, is the context's reusable device buffer); unpack: enqueued
 * on `stream` (NULL = the context's).
 * No counterpart in the reference. */
p2z_status p2z_pack_by_hits_device(p2z_context *ctx, const p2z_config *cfg, const void *d_trk_in,
                                   const void *d_hits_in, const uint32_t *d_mask_in, void *d_trk_out,
                                   void *d_hits_out, uint32_t *d_mask_out, int64_t *d_perm, void *stream);
p2z_status p2z_unpack_tracks_device(p2z_context *ctx, const p2z_config *cfg, const int64_t *d_perm,
                                    const void *d_trk_packed, void *d_trk_out, void *stream);

/* One measured launch configuration. */
typedef struct p2z_tune_entry {
  int32_t bsize;          /* 8, 16, 32, 64 */
  int32_t layout;         /* p2z_layout */
  int32_t schedule;       /* P2Z_SCHED_FLAT, _PER_EVENT, _PERSISTENT or _STAGED */
  int32_t block_threads;  /* 32 .. 256 */
  int32_t threads_per_track; /* 1 or 2 */
  uint32_t flags;         /* P2Z_FLAG_SORT_WINDOWS when the row sorted windows, else 0 */
  double ms;              /* mean device time of one pass */
  double updates_per_s;   /* present-hit updates per second */
} p2z_tune_entry;

/* Autotuner: measures one pass of cfg's work (its update kind and flags, one
 * iteration) on the caller's device data under every combination of bsize
 * {8,16,32,64} x layout {AOSOA, SOA} x schedule {FLAT, PERSISTENT, PER_EVENT
 * when nevts <= 4096, and STAGED at bsize 32 AOSOA} x block_threads
 * {32,64,128,256} x threads_per_track {1, and 2 where the update kind and
 * schedule have it} x, for masked runs on the FLAT and PERSISTENT schedules,
 * window sorting {off, P2Z_FLAG_SORT_WINDOWS}, each the mean
 * of `reps` passes (0 -> 3) after one warm-up pass.  The inputs are converted
 * to each candidate's bsize and layout with p2z_relayout_device into scratch
 * buffers the call allocates and frees (about twice the input size); the
 * caller's buffers are only read.  Results: the number of configurations
 * measured in *n_entries, the first max_entries of them in `entries` (may be
 * NULL when max_entries is 0), the fastest in *best.
 * Side effect: for every (bsize, layout) measured, the context remembers the
 * fastest schedule, block size, threads per track and window sorting, and
 * later runs with block_threads = 0, schedule = AUTO or threads_per_track = 0
 * and the same update, flags, bsize, layout and masking use them (window
 * sorting when the schedule is AUTO).  A different bsize or layout is a different data layout, which only
 * the caller can adopt (p2z_relayout_device).  Synchronous. */
p2z_status p2z_autotune(p2z_context *ctx, const p2z_config *cfg, const void *d_trk_in, const void *d_hits,
                        const uint32_t *d_hit_mask, int reps, p2z_tune_entry *entries, int max_entries,
                        int *n_entries, p2z_tune_entry *best);

/* ---- inputs (prepareTracks / prepareHits) ----------------------------------- */

/* Seed structs, layout-identical to the reference's ATRK and AHIT
 * (src/propagate-toz-test_OMP.cpp:57-67). */
typedef struct p2z_atrk { float par[6]; float cov[21]; int32_t q; } p2z_atrk;
typedef struct p2z_ahit { float pos[3]; float cov[6]; } p2z_ahit;

/* The reference's input preparation: srand(1) (:715-718), then prepareTracks
 * (:243-263) and prepareHits (:265-293), consuming the C library's rand()
 * stream in the same order through the same polar-method randn (:127-145).
 * Every element is multiplied by (1 + smear*N(0,1)); covariance elements are
 * further multiplied by cov_scale (the reference uses 100); charge is copied.
 * Layer l uses hit seed l; nseeds < nlayer is P2Z_BAD_ARG (the reference exits).
 * With smear = 1e-7 and cov_scale = 100 the output is bit-identical to the
 * reference's.  Host memory; trk_out holds nevts*ntrks/bsize MPTRK, hits_out
 * nlayer*nevts*ntrks/bsize MPHIT.  Uses a private generator state (the global
 * rand() state is not touched) so concurrent calls are safe. */
p2z_status p2z_prepare(const p2z_atrk *seed, const p2z_ahit *hit_seeds, int nseeds, int bsize, int64_t nevts,
                       int64_t ntrks, int nlayer, double smear, double cov_scale, void *trk_out, void *hits_out);

/* The reference's random stream, resumable: the C library's rand() after
 * srand(seed) (glibc's additive generator, restated) and the reference's
 * polar-method randn (src/propagate-toz-test_OMP.cpp:127-145), whose second
 * variate of a pair is kept for the next call.  A plain struct: copy it to
 * fork the stream.  p2z_prepare is p2z_ref_rng_seed(1), p2z_prepare_tracks,
 * p2z_prepare_hits on one stream, as the reference's main calls
 * prepareTracks then prepareHits (:715-720). */
typedef struct p2z_ref_rng {
  uint32_t ring[31];     /* the generator's last 31 words */
  int32_t have_second;   /* randn holds the second variate of a pair */
  int64_t next;          /* index of the next word */
  float second;
  int32_t reserved;
} p2z_ref_rng;
void p2z_ref_rng_seed(p2z_ref_rng *g, uint32_t seed);  /* srand(seed) */
int32_t p2z_ref_rng_rand(p2z_ref_rng *g);               /* rand() */
float p2z_ref_rng_randn(p2z_ref_rng *g);                /* randn(0, 1) */
/* prepareTracks (:243-263) on the stream g: nevts*ntrks/bsize MPTRK (host),
 * every element times (1 + smear*randn), covariance also times cov_scale. */
p2z_status p2z_prepare_tracks(p2z_ref_rng *g, const p2z_atrk *seed, int bsize, int64_t nevts, int64_t ntrks,
                              double smear, double cov_scale, void *trk_out);
/* prepareHits (:265-293) on the stream g: nlayer*nevts*ntrks/bsize MPHIT
 * (host), layer l from hit seed l; nseeds < nlayer is P2Z_BAD_ARG. */
p2z_status p2z_prepare_hits(p2z_ref_rng *g, const p2z_ahit *hit_seeds, int nseeds, int bsize, int64_t nevts,
                            int64_t ntrks, int nlayer, double smear, void *hits_out);

/* p2z_prepare generated on the device into device buffers (AOSOA, bsize
 * batches): the same words as p2z_prepare, for callers whose tracks and hits
 * live on the GPU.  The reference's rand() stream is split into chunks whose
 * starting states are computed by jumping its additive generator ahead, the
 * polar method's accepted attempts are counted per chunk and prefix-summed,
 * and every variate is written to its word in parallel.  The variate's log is
 * correctly rounded where p2z_prepare calls the C library's logf (which
 * differs in the last place for ~0.3% of variates; that changed no output
 * word on 200M variates, and the tests compare the outputs word for word).
 * Scratch from the context.  Enqueued on `stream` (NULL = the context's
 * stream); returns when the output is complete.  No counterpart in the
 * reference, which prepares on the host (src/propagate-toz-test_OMP.cpp:
 * 243-293). */
p2z_status p2z_prepare_device(p2z_context *ctx, const p2z_atrk *seed, const p2z_ahit *hit_seeds, int nseeds,
                              int bsize, int64_t nevts, int64_t ntrks, int nlayer, double smear, double cov_scale,
                              void *d_trk_out, void *d_hits_out, void *stream);

/* Physics workload generator (no counterpart in the reference): tracks of
 * charge +-1, pT log-uniform in [pt_min, pt_max] GeV, phi ~ U(-pi, pi),
 * eta ~ U(eta_min, eta_max), vertex z ~ N(0, sigma_vz); covariance
 * diag(sigma) * random correlation (|rho| <= rho_max, positive definite) * diag(sigma)
 * with sigma = (sig_xy, sig_xy, sig_z, rel_sig_ipt*ipt, sig_phi, sig_theta); the
 * initial parameters are the truth smeared with that covariance.  Hits on nlayer
 * planes z_first..z_last at the true helix point (the propagateToZ helix with
 * the same kfact, evaluated in FP64) plus Gaussian noise (hit_sig_xy, hit_sig_z)
 * with a diagonal 3x3 covariance.  Counter-based RNG: output depends only on
 * (seed, track index), independent of threading.  Uniform or uneven events
 * (event_ntrks != NULL); hit_mask (optional) receives all-present masks for
 * real tracks and 0 for padding slots. */
typedef struct p2z_physics_params {
  uint64_t seed;
  double pt_min, pt_max, eta_min, eta_max, sigma_vz;
  double sig_xy, sig_z, rel_sig_ipt, sig_phi, sig_theta, rho_max;
  double z_first, z_last;
  double hit_sig_xy, hit_sig_z;
  float kfact;  /* 0 -> default */
  int32_t nthreads; /* host threads; 0 -> all */
} p2z_physics_params;
void p2z_physics_defaults(p2z_physics_params *p);
p2z_status p2z_generate_physics(const p2z_physics_params *p, const p2z_config *cfg, void *trk_out, void *hits_out,
                                uint32_t *hit_mask);

/* The same physics sample generated on the device into device buffers (AOSOA
 * layout): the same per-slot computation in the same double expressions, so
 * the output equals p2z_generate_physics's except where CUDA's and the C
 * library's log/exp/sin/cos/tan/atan round a double differently (a float
 * output then differs by one unit in the last place; rare).  p->nthreads is
 * ignored.  Enqueued on `stream` (NULL = the context's stream); returns when
 * the generation is complete.  No counterpart in the reference, which prepares
 * its inputs on the host (src/propagate-toz-test_OMP.cpp:243-293). */
p2z_status p2z_generate_physics_device(p2z_context *ctx, const p2z_physics_params *p, const p2z_config *cfg,
                                       void *d_trk_out, void *d_hits_out, uint32_t *d_hit_mask, void *stream);

/* Drop layers from a hit mask (no counterpart in the reference): each real
 * track (mask != 0) keeps a contiguous run of L layers starting at layer 0 with
 * L uniform in [min_hits, max_hits], then loses each layer independently with
 * probability drop_prob as long as at least min_hits remain.  Deterministic in
 * (seed, slot). */
p2z_status p2z_mask_layers(uint32_t *hit_mask, int64_t nslots, int nlayer, int min_hits, int max_hits,
                           double drop_prob, uint64_t seed);
/* The same on a device mask array (bit-identical to p2z_mask_layers: the draws
 * use no library function), enqueued on `stream` (NULL = the context's). */
p2z_status p2z_mask_layers_device(p2z_context *ctx, uint32_t *d_hit_mask, int64_t nslots, int nlayer, int min_hits,
                                  int max_hits, double drop_prob, uint64_t seed, void *stream);

/* ---- validation block ------------------------------------------------------- */

/* Accumulators of the reference's printed validation block
 * (src/propagate-toz-test_OMP.cpp:758-876). */
typedef struct p2z_validation {
  double avgx, avgy, avgz, avgdx, avgdy, avgdz, avgpt, avgphi, avgtheta;
  double stdx, stdy, stdz, stddx, stddy, stddz;
  int64_t nnans, nfail, ngood;
} p2z_validation;

/* Compute the block over nevts*ntrks output tracks against the last-layer
 * seed hit (hx, hy, hz), with the reference's NaN test, its "fail" window
 * (pt~12, phi~1.3, theta~2.8, :784-795) and its divisions by ngood. */
p2z_status p2z_validate(const void *trk_out, int bsize, int64_t nevts, int64_t ntrks, const float hit_last[3],
                        p2z_validation *v);
/* The same block for work split over several processes (one event shard
 * each): pass 1 (means == NULL) accumulates the sums and counts of the tracks
 * given; after the caller sums pass-1 partials over all shards (an all-reduce
 * of the doubles and counts), p2z_validate_means gives the global means; pass 2
 * (means != NULL) accumulates the squared deviations from them; summing those
 * and calling p2z_validate_combine yields the block of the whole sample.  This
 * is the reference's two-pass computation (:758-864) with the passes'
 * accumulators reduced across shards between them.  No counterpart in the
 * reference (single process). */
typedef struct p2z_validation_partial {
  double sum[9];  /* x, y, z, dx/x, dy/y, dz/z, pt, phi, theta (pass 1) */
  double sq[6];   /* squared deviations of x, y, z, dx/x, dy/y, dz/z (pass 2) */
  int64_t nnans, nfail, ngood;
} p2z_validation_partial;
p2z_status p2z_validate_partial(const void *trk_out, int bsize, int64_t nevts, int64_t ntrks, const float hit_last[3],
                                const double means[6], p2z_validation_partial *acc);
void p2z_validate_means(const p2z_validation_partial *pass1, double means[6]);
p2z_status p2z_validate_combine(const p2z_validation_partial *pass1, const p2z_validation_partial *pass2,
                                p2z_validation *v);
/* The same two passes over DEVICE-resident output tracks (AOSOA, bsize
 * batches, nevts*ntrks tracks), reduced on the GPU: every track's values and
 * selection are computed exactly as in p2z_validate (the same double
 * expressions, so the same counts); the sums are taken in a fixed tree order
 * (deterministic from run to run) instead of the reference's sequential one,
 * so they agree with the host's to about 1e-15 relative.  The per-block
 * partials live in the context's scratch.  Enqueued on `stream` (NULL = the
 * context's stream); returns when the results are on the host.  Replaces the
 * host loop of the reference's validation block (:758-864) for outputs that
 * are still on the device; p2z_validate_partial_device is the per-shard form. */
p2z_status p2z_validate_device(p2z_context *ctx, const void *d_trk_out, int bsize, int64_t nevts, int64_t ntrks,
                               const float hit_last[3], p2z_validation *v, void *stream);
p2z_status p2z_validate_partial_device(p2z_context *ctx, const void *d_trk_out, int bsize, int64_t nevts,
                                       int64_t ntrks, const float hit_last[3], const double means[6],
                                       p2z_validation_partial *acc, void *stream);
/* Print it with the reference's exact format (:866-876) to stdout. */
void p2z_print_validation(const p2z_validation *v);
/* The per-track dump of the reference's DUMP_OUTPUT build
 * (src/propagate-toz-test_CUDA_v4.cu:1012-1143): for every track that passes
 * the validation's NaN test and window (as in p2z_validate), one "%f" line
 * with its output x, y, z in output_x.txt, output_y.txt, output_z.txt and its
 * input x, y, z in input_x.txt, input_y.txt, input_z.txt, in the directory
 * `dir` (NULL or "" = the current directory).  Host arrays.  The tracks are
 * selected against the last-layer seed hit, as p2z_validate does. */
p2z_status p2z_dump_tracks(const void *trk_in, const void *trk_out, int bsize, int64_t nevts, int64_t ntrks,
                           const float hit_last[3], const char *dir);
/* The machine-readable line of the reference (:756), parsed by its tools
 * (tools/compare.py:12): "formatted NITER nevts ntrks bsize nb wall 0 setup nthreads". */
void p2z_print_formatted(int niter, int64_t nevts, int64_t ntrks, int bsize, double wall_s, double setup_s,
                         int nthreads);

/* ---- serving: continuous batching (no counterpart in the reference) -------- */

/* A server owns a device "slot ring" sized by a memory budget: parallel ring
 * buffers of track batches, output batches, hit batches and masks indexed by
 * one batch number, so every admitted event occupies one contiguous range of
 * batches.  A scheduler thread admits submitted events in arrival order while
 * ring space allows (copying their inputs host->device on a copy stream),
 * launches every admitted-but-not-yet-launched event together as one group
 * (the persistent work-queue kernel over the group's contiguous slot range),
 * copies each event's tracks back on its own completion event and frees ring
 * space in completion order.  Events that arrive while a group is on the GPU
 * are copied in meanwhile and form the next group as soon as the number of
 * groups in flight drops below max_inflight: copies, kernels and read-backs of
 * different events overlap.  Per-track arithmetic does not depend on the
 * group, so an event's result is the same alone and in any mix. */
typedef struct p2z_server p2z_server;

typedef struct p2z_server_config {
  int32_t abi_version;         /* P2Z_ABI_VERSION */
  int32_t bsize;               /* AOSOA width of the submitted events */
  int32_t nlayer;
  int32_t update;              /* p2z_update_kind */
  uint32_t flags;              /* P2Z_FLAG_ACCURATE_TRIG / REFERENCE_ROUNDING / FULL_HITS; any other
                                  flag: p2z_server_create returns P2Z_UNSUPPORTED */
  float kfact;                 /* 0 -> P2Z_KFACT_DEFAULT */
  int64_t device_budget_bytes; /* size of the slot ring */
  int32_t max_inflight;        /* launch groups on the GPU at once; 0 -> 2 */
  int32_t block_threads;       /* 0 -> 128 */
} p2z_server_config;

typedef struct p2z_request_info {
  double submit_s, admit_s, launch_s, done_s; /* host steady-clock seconds */
  int64_t ntrks;
  int64_t updates;       /* present hits */
  int32_t group_events;  /* events launched together with this one */
  int32_t status;        /* p2z_status of the request */
} p2z_request_info;

p2z_status p2z_server_create(int device, const p2z_server_config *cfg, p2z_server **out);
/* Waits for every submitted event, then releases the server. */
p2z_status p2z_server_destroy(p2z_server *srv);
/* One event of ntrks tracks: trk_in holds ceil(ntrks/bsize) MPTRK batches,
 * hits nlayer MPHIT per batch, hit_mask (optional) one word per slot; the
 * updated tracks go to trk_out.  Host buffers (page-locked for asynchronous
 * copies) must stay valid until the request completes.  Returns at once;
 * P2Z_OOM if the event alone exceeds the ring. */
p2z_status p2z_server_submit(p2z_server *srv, const void *trk_in, const void *hits, const uint32_t *hit_mask,
                             int64_t ntrks, void *trk_out, int64_t *id);
/* P2Z_OK and the request's timings once it has completed, else P2Z_NOT_READY.
 * A completed request is released once poll or wait has reported it. */
p2z_status p2z_server_poll(p2z_server *srv, int64_t id, p2z_request_info *info);
/* Blocks until the request completes or timeout_s passes (P2Z_TIMEOUT). */
p2z_status p2z_server_wait(p2z_server *srv, int64_t id, double timeout_s, p2z_request_info *info);
/* Seconds on the server's clock (the one the request timings use). */
double p2z_server_now(const p2z_server *srv);
/* Load replay for measurements: submits nreq events at the given arrival
 * times (seconds from the call), waits for all of them and fills infos. */
p2z_status p2z_server_replay(p2z_server *srv, int64_t nreq, const void *const *trk_in, const void *const *hits,
                             const uint32_t *const *hit_mask, const int64_t *ntrks, void *const *trk_out,
                             const double *arrival_s, p2z_request_info *infos);

/* ---- measured roofline denominators (no counterpart in the reference) ------ */

/* Throughputs of the current GPU and its host link, as the benchmark divides by:
 * FP32 fused multiply-adds (independent chains on every lane of every SM, 64
 * warps per SM) issued as scalar FFMA and as paired FP32x2 FFMA2, in TFLOP/s
 * (an FMA is 2 flops); pinned host->device, device->host and both at once
 * (two streams; the sum of the two directions), in GB/s, for one copy of
 * copy_bytes (0 -> 1 GiB) each way.  Best of `reps` (0 -> 5) after one
 * warm-up.  Allocates its own buffers; changes no GPU setting.  device < 0:
 * the current device.  Synchronous. */
typedef struct p2z_peaks {
  double fp32_ffma_tflops;
  double fp32_ffma2_tflops;
  double h2d_gbs, d2h_gbs, bidir_gbs;
  int64_t copy_bytes;
  int32_t sms;
} p2z_peaks;
p2z_status p2z_measure_peaks(int device, size_t copy_bytes, int reps, p2z_peaks *out);

/* ---- host memory helpers ---------------------------------------------------- */

/* Page-locked host allocation (cudaHostAlloc) for fast asynchronous copies. */
p2z_status p2z_host_alloc(void **ptr, size_t bytes);
p2z_status p2z_host_free(void *ptr);

/* Device memory on the context's device, for callers without the CUDA
 * runtime of their own (the typed C++ layer, include/p2z_types.hpp):
 * cudaMalloc / cudaFree, and a copy in any direction between host and device
 * pointers (unified addressing) that returns when the copy is complete.  No
 * counterpart in the reference, whose GPU builds call the CUDA runtime in main
 * (src/propagate-toz-test_CUDA_v4.cu:921-947). */
p2z_status p2z_device_alloc(p2z_context *ctx, void **d_ptr, size_t bytes);
p2z_status p2z_device_free(p2z_context *ctx, void *d_ptr);
p2z_status p2z_copy(p2z_context *ctx, void *dst, const void *src, size_t bytes);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#pragma pop_macro("N")
#pragma pop_macro("smear")
#pragma pop_macro("nthreads")
#pragma pop_macro("NITER")
#pragma pop_macro("nb")
#pragma pop_macro("nlayer")
#pragma pop_macro("ntrks")
#pragma pop_macro("nevts")
#pragma pop_macro("bsize")

#endif /* P2Z_H */
