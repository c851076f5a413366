// p2z_api.cu -- the extern "C" boundary (include/p2z.h): contexts, the hot-path
// run entry points, launch scheduling (flat / per-event / persistent replayed
// as a CUDA graph) and host<->device copy pipelining.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "p2z.h"
#include "p2z_kernels.cuh"

// p2z_run: the host<->device copies and the kernels are pipelined over at most
// this many chunks (alternating between two streams).  Measured on one B200 for
// the 1000-event sample: 8 chunks 108.4 ms, 16 107.8 ms, 32 108.1-108.5 ms.
#ifndef P2Z_RUN_MAX_CHUNKS
#define P2Z_RUN_MAX_CHUNKS 16
#endif
// P2Z_FLAG_PER_EVENT_STREAMS: streams the per-event launches are spread over.
constexpr int kEventStreams = 10;
// Masked runs with P2Z_FLAG_SORT_WINDOWS: slots per sorted window.
// A warp's 32 tracks take as many steps as the longest of them; with hit
// counts of 5-20 per track, 32 slots taken in stored order keep 60% of the
// lane-steps busy; sorted by hit count, windows of 64, 128 and 256 slots keep
// 74%, 85% and 92%.  A sorted warp's loads reach as many batches of 32 as the
// window holds, which costs per step: measured on one B200 (2000-event
// sample, persistent schedule) 1.725, 1.668 and 2.189 ms against 1.894 ms in
// stored order, so the window is 128 slots.
#ifndef P2Z_SORT_WINDOW
#define P2Z_SORT_WINDOW 128
#endif

namespace p2z {
cudaError_t launch_step(int bsize, float *trk, const float *hits, int64_t nslots, int nlayer, int layer, int what,
                        float kfact, cudaStream_t st);
}

using namespace p2z;

namespace {

std::mutex g_err_mu;
std::string g_last_error;  // failures with no context

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
};

struct GraphKey {
  RunArgs args;
  int bsize, upd, sc, block, grid, kind, tpt;
  bool masked, soa;
  bool operator==(const GraphKey &o) const { return std::memcmp(this, &o, sizeof(GraphKey)) == 0; }
};

// Launch shape p2z_autotune measured fastest for one kind of run.
struct Tuned {
  int upd, sc, B;
  bool soa, masked;
  int block, schedule, tpt;
  bool sort;  // P2Z_FLAG_SORT_WINDOWS
};

}  // namespace

struct p2z_context {
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy[2] = {nullptr, nullptr};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr, ev3 = nullptr;
  cudaEvent_t join[2] = {nullptr, nullptr};
  unsigned int *d_status = nullptr;         // device status word
  unsigned int *h_status = nullptr;         // page-locked copy of it (p2z_run)
  unsigned long long *d_queue = nullptr;    // 2 persistent work counters (one per copy stream)
  DevBuf trk, hits, out, mask, valid;       // p2z_run buffers / internal masks
  // what `mask` holds as an internal padding mask: (mask address, bsize, nlayer, the events' track
  // counts); empty when it holds anything else (a caller's mask copied by p2z_run)
  std::vector<int64_t> mask_key;
  DevBuf aux;                               // scratch of the validation reduction
  DevBuf perm;                              // sorted-window permutation (masked runs)
  bool has_graph = false;
  GraphKey gkey;
  cudaGraphExec_t gexec = nullptr;
  std::vector<Tuned> tuned;                 // p2z_autotune results
  cudaStream_t ev_streams[kEventStreams] = {};  // P2Z_FLAG_PER_EVENT_STREAMS (created on first use)
  cudaEvent_t ev_fork = nullptr, ev_join[kEventStreams] = {};
  // p2z_run's copy/kernel pipeline recorded as a graph (page-locked host buffers),
  // with what it was recorded for and what it enqueues
  cudaGraphExec_t run_exec = nullptr;
  std::vector<int64_t> run_key;
  int run_launches = 0;
  int64_t run_h2d = 0, run_d2h = 0;
  std::string last_error;
};

namespace {

p2z_status fail(p2z_context *ctx, p2z_status st, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (ctx) {
    ctx->last_error = buf;
  } else {
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_last_error = buf;
  }
  return st;
}

#define P2Z_CUDA(ctx, call)                                                                          \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess)                                                                           \
      return fail((ctx), e_ == cudaErrorMemoryAllocation ? P2Z_OOM : P2Z_CUDA_ERROR, "%s: %s (%s:%d)", \
                  #call, cudaGetErrorString(e_), __FILE__, __LINE__);                                \
  } while (0)

p2z_status ensure(p2z_context *ctx, DevBuf &b, size_t bytes) {
  if (b.bytes >= bytes) return P2Z_OK;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
  if (bytes == 0) return P2Z_OK;
  cudaError_t e = cudaMalloc(&b.p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, P2Z_OOM, "cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
  }
  b.bytes = bytes;
  return P2Z_OK;
}

bool valid_bsize(int b) { return b == 8 || b == 16 || b == 32 || b == 64; }

// Validated view of a config.
struct Plan {
  int B = 0;
  int nlayer = 0;
  int niter = 1;
  float kfact = 0.f;
  int upd = 0;
  int sc = SC_FAST;
  int schedule = P2Z_SCHED_FLAT;
  int block = 0;
  int tpt = 1;               // threads per track
  uint32_t flags = 0;
  int64_t nbatches = 0;
  int64_t nslots = 0;
  bool uneven = false;
  bool soa = false;          // P2Z_LAYOUT_SOA
  std::vector<int64_t> ev_slot_begin;  // nevts + 1 entries
  const int64_t *event_ntrks = nullptr;  // uneven: the caller's tracks per event
};

p2z_status make_plan(p2z_context *ctx, const p2z_config *cfg, Plan &pl) {
  if (!cfg) return fail(ctx, P2Z_BAD_ARG, "config is NULL");
  if (cfg->abi_version != P2Z_ABI_VERSION)
    return fail(ctx, P2Z_BAD_ARG, "abi_version %d != %d", cfg->abi_version, P2Z_ABI_VERSION);
  if (!valid_bsize(cfg->bsize)) return fail(ctx, P2Z_UNSUPPORTED, "bsize %d not in {8,16,32,64}", cfg->bsize);
  if (cfg->nlayer < 1 || cfg->nlayer > 32) return fail(ctx, P2Z_BAD_ARG, "nlayer %d not in 1..32", cfg->nlayer);
  if (cfg->nevts < 0) return fail(ctx, P2Z_BAD_ARG, "nevts %lld < 0", (long long)cfg->nevts);
  if (cfg->update < P2Z_UPDATE_V2 || cfg->update > P2Z_UPDATE_F64)
    return fail(ctx, P2Z_BAD_ARG, "update kind %d unknown", cfg->update);
  if (cfg->schedule < P2Z_SCHED_AUTO || cfg->schedule > P2Z_SCHED_STAGED)
    return fail(ctx, P2Z_BAD_ARG, "schedule %d unknown", cfg->schedule);
  if (cfg->block_threads != 0 && (cfg->block_threads < 32 || cfg->block_threads > 256 || cfg->block_threads % 32))
    return fail(ctx, P2Z_BAD_ARG, "block_threads %d not a multiple of 32 in 32..256", cfg->block_threads);
  if (cfg->layout != P2Z_LAYOUT_AOSOA && cfg->layout != P2Z_LAYOUT_SOA)
    return fail(ctx, P2Z_BAD_ARG, "layout %d unknown", cfg->layout);
  if (cfg->niter < 0) return fail(ctx, P2Z_BAD_ARG, "niter %d < 0", cfg->niter);
  if (!std::isfinite(cfg->kfact)) return fail(ctx, P2Z_BAD_ARG, "kfact is not finite");
  pl.soa = cfg->layout == P2Z_LAYOUT_SOA;
  pl.B = cfg->bsize;
  pl.nlayer = cfg->nlayer;
  pl.niter = cfg->niter > 0 ? cfg->niter : 1;
  pl.kfact = cfg->kfact != 0.f ? cfg->kfact : (float)(100. / (-0.299792458 * 3.8112));
  pl.upd = cfg->update;
  pl.flags = cfg->flags;
  constexpr uint32_t kKnownFlags = P2Z_FLAG_CHECK_INPUTS | P2Z_FLAG_STRICT | P2Z_FLAG_NO_GRAPH |
                                   P2Z_FLAG_ACCURATE_TRIG | P2Z_FLAG_FULL_HITS | P2Z_FLAG_REFERENCE_ROUNDING |
                                   P2Z_FLAG_PER_EVENT_STREAMS | P2Z_FLAG_SORT_WINDOWS;
  if (cfg->flags & ~kKnownFlags) return fail(ctx, P2Z_BAD_ARG, "unknown flag bits 0x%x", cfg->flags & ~kKnownFlags);
  if (cfg->flags & P2Z_FLAG_REFERENCE_ROUNDING) {
    if (cfg->update != P2Z_UPDATE_V2)
      return fail(ctx, P2Z_UNSUPPORTED, "P2Z_FLAG_REFERENCE_ROUNDING applies to P2Z_UPDATE_V2 only");
    pl.upd = UPDK_V2_REF;
  }
  pl.sc = (cfg->flags & P2Z_FLAG_ACCURATE_TRIG) ? SC_ACCURATE : SC_FAST;
  pl.block = cfg->block_threads ? cfg->block_threads : 128;
  if (cfg->threads_per_track < 0 || cfg->threads_per_track > 2)
    return fail(ctx, P2Z_UNSUPPORTED, "threads_per_track %d not in {0, 1, 2}", cfg->threads_per_track);
  if (cfg->threads_per_track == 2 && pl.upd != UPDK_V2)
    return fail(ctx, P2Z_UNSUPPORTED, "threads_per_track 2 applies to P2Z_UPDATE_V2 without "
                                      "P2Z_FLAG_REFERENCE_ROUNDING only");
  if (cfg->threads_per_track == 2 && cfg->schedule == P2Z_SCHED_STAGED)
    return fail(ctx, P2Z_UNSUPPORTED, "the staged schedule has one thread per track");
  pl.tpt = cfg->threads_per_track == 2 ? 2 : 1;
  pl.ev_slot_begin.assign((size_t)cfg->nevts + 1, 0);
  if (cfg->event_ntrks) {
    pl.uneven = true;
    int64_t nb = 0;
    for (int64_t e = 0; e < cfg->nevts; ++e) {
      const int64_t n = cfg->event_ntrks[e];
      if (n < 0) return fail(ctx, P2Z_BAD_ARG, "event_ntrks[%lld] = %lld < 0", (long long)e, (long long)n);
      pl.ev_slot_begin[e] = nb * pl.B;
      nb += (n + pl.B - 1) / pl.B;
    }
    pl.nbatches = nb;
    pl.event_ntrks = cfg->event_ntrks;
    pl.ev_slot_begin[cfg->nevts] = nb * pl.B;
  } else {
    if (cfg->ntrks < 0 || cfg->ntrks % cfg->bsize)
      return fail(ctx, P2Z_BAD_ARG, "ntrks %lld is not a non-negative multiple of bsize %d", (long long)cfg->ntrks,
                  cfg->bsize);
    pl.nbatches = cfg->nevts * (cfg->ntrks / cfg->bsize);
    for (int64_t e = 0; e <= cfg->nevts; ++e) pl.ev_slot_begin[e] = e * cfg->ntrks;
  }
  pl.nslots = pl.nbatches * pl.B;
  pl.schedule = cfg->schedule;
  return P2Z_OK;
}

cudaError_t dispatch(const LaunchSpec &s, cudaStream_t st) {
  switch (s.upd) {
    case UPDK_V2: return launch_v2(s, st);
    case UPDK_V2_COMP: return launch_v2_comp(s, st);
    case UPDK_3X3_F64: return launch_3x3_f64(s, st);
    case UPDK_3X3_COMP: return launch_3x3_comp(s, st);
    case UPDK_F64: return launch_f64(s, st);
    case UPDK_V2_REF: return launch_v2_ref(s, st);
  }
  return cudaErrorInvalidValue;
}

int occupancy(const LaunchSpec &s) {
  switch (s.upd) {
    case UPDK_V2: return occupancy_v2(s);
    case UPDK_V2_COMP: return occupancy_v2_comp(s);
    case UPDK_3X3_F64: return occupancy_3x3_f64(s);
    case UPDK_3X3_COMP: return occupancy_3x3_comp(s);
    case UPDK_F64: return occupancy_f64(s);
    case UPDK_V2_REF: return occupancy_v2_ref(s);
  }
  return 0;
}

// Writes masks for uneven events: all layers for real lanes, 0 for padding.
__global__ void k_fill_mask(uint32_t *mask, const uint8_t *valid, int64_t nslots, int B, uint32_t all) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslots) return;
  mask[s] = ((int)(s % B) < (int)valid[s / B]) ? all : 0u;
}

// Sum of popcounts of the masks (track-layer updates requested).
__global__ void k_count_updates(const uint32_t *mask, int64_t nslots, uint32_t all, unsigned long long *out) {
  unsigned long long acc = 0;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nslots; s += (int64_t)gridDim.x * blockDim.x)
    acc += __popc(mask[s] & all);
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(out, acc);
}

uint32_t all_layers(int nlayer) { return nlayer >= 32 ? 0xffffffffu : ((1u << nlayer) - 1u); }

// One CTA per window of `win` slots of [s0, s1): a counting sort of the
// window's slots by hit count, most hits first, written as the within-window
// offset of the slot each rank processes (perm[window base + rank]).  Ranks
// of equal hit count are assigned by shared-memory atomics, so which thread
// processes which of them varies from run to run; every track's arithmetic
// is independent of its thread, so the results do not.
__global__ void __launch_bounds__(P2Z_SORT_WINDOW) k_sort_windows(const uint32_t *__restrict__ mask, uint8_t *perm,
                                                                  int64_t s0, int64_t s1, int win, uint32_t all) {
  __shared__ int hist[33];
  __shared__ int start[33];
  const int i = threadIdx.x;
  const int64_t base = s0 + (int64_t)blockIdx.x * win;
  const int n = (int)min((int64_t)win, s1 - base);
  if (i < 33) hist[i] = 0;
  __syncthreads();
  int key = 0, pos = 0;
  if (i < n) {
    key = 32 - __popc(__ldg(mask + base + i) & all);  // 0 = all 32 layers present
    pos = atomicAdd(&hist[key], 1);
  }
  __syncthreads();
  if (i == 0) {
    int acc = 0;
    for (int k = 0; k < 33; ++k) {
      start[k] = acc;
      acc += hist[k];
    }
  }
  __syncthreads();
  if (i < n) perm[base + start[key] + pos] = (uint8_t)i;
}

// The streams and events P2Z_FLAG_PER_EVENT_STREAMS spreads per-event launches
// over, created on first use.
p2z_status event_streams(p2z_context *ctx) {
  if (ctx->ev_fork) return P2Z_OK;
  for (int i = 0; i < kEventStreams; ++i) {
    P2Z_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->ev_streams[i], cudaStreamNonBlocking));
    P2Z_CUDA(ctx, cudaEventCreateWithFlags(&ctx->ev_join[i], cudaEventDisableTiming));
  }
  P2Z_CUDA(ctx, cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
  return P2Z_OK;
}

// True for page-locked host memory (cudaHostAlloc / cudaHostRegister).
bool page_locked(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Enqueue the hot-path launches of one pass over slots [s0, s1) on st.
// queue: the persistent work counter to use.
p2z_status enqueue_pass(p2z_context *ctx, const Plan &pl, const RunArgs &base, int64_t s0, int64_t s1,
                        int schedule, cudaStream_t st, unsigned long long *queue, int *launches) {
  LaunchSpec spec;
  spec.args = base;
  spec.args.queue = queue;
  spec.bsize = pl.B;
  spec.soa = pl.soa;
  spec.args.ws = pl.nslots;
  spec.upd = pl.upd;
  spec.sc = pl.sc;
  spec.masked = base.mask != nullptr;
  spec.block = pl.block;
  spec.grid = 0;
  spec.tpt = pl.tpt;
  // Launches of at most 4 warps per SM leave each scheduler about one warp, with
  // nothing to run while it waits for a layer's hits from DRAM: those launches
  // ask L2 for their batches' hit blocks first (AOSOA).
  const int64_t small_slots = (int64_t)ctx->num_sms * 4 * 32 / pl.tpt;
  auto prefetch_for = [&](int64_t n) { return (!pl.soa && n <= small_slots) ? 1 : 0; };
  if (pl.tpt != 1 && schedule == P2Z_SCHED_STAGED)
    return fail(ctx, P2Z_UNSUPPORTED, "the staged schedule has one thread per track");
  if (schedule == P2Z_SCHED_PER_EVENT) {
    spec.kind = KIND_FLAT;
    const bool spread = (pl.flags & P2Z_FLAG_PER_EVENT_STREAMS) != 0;
    if (spread) {
      p2z_status r = event_streams(ctx);
      if (r != P2Z_OK) return r;
      P2Z_CUDA(ctx, cudaEventRecord(ctx->ev_fork, st));
      for (int i = 0; i < kEventStreams; ++i) P2Z_CUDA(ctx, cudaStreamWaitEvent(ctx->ev_streams[i], ctx->ev_fork, 0));
    }
    const int64_t nev = (int64_t)pl.ev_slot_begin.size() - 1;
    int k = 0;
    for (int64_t e = 0; e < nev; ++e) {
      const int64_t a = std::max(s0, pl.ev_slot_begin[e]), b = std::min(s1, pl.ev_slot_begin[e + 1]);
      if (b <= a) continue;
      spec.args.slot_begin = a;
      spec.args.slot_end = b;
      spec.args.l2_prefetch = prefetch_for(b - a);
      P2Z_CUDA(ctx, dispatch(spec, spread ? ctx->ev_streams[k++ % kEventStreams] : st));
      ++*launches;
    }
    if (spread) {
      for (int i = 0; i < kEventStreams; ++i) {
        P2Z_CUDA(ctx, cudaEventRecord(ctx->ev_join[i], ctx->ev_streams[i]));
        P2Z_CUDA(ctx, cudaStreamWaitEvent(st, ctx->ev_join[i], 0));
      }
    }
    return P2Z_OK;
  }
  spec.args.slot_begin = s0;
  spec.args.slot_end = s1;
  if (s1 <= s0) return P2Z_OK;
  spec.args.l2_prefetch = prefetch_for(s1 - s0);  // (the staged kernel stages its hits itself)
  // masked flat and persistent runs: process each window's slots in order of hit count
  const bool sort = spec.masked && (pl.flags & P2Z_FLAG_SORT_WINDOWS) &&
                    (schedule == P2Z_SCHED_FLAT || schedule == P2Z_SCHED_PERSISTENT);
  if (sort) {
    p2z_status r = ensure(ctx, ctx->perm, (size_t)pl.nslots);
    if (r != P2Z_OK) return r;
    spec.args.perm = (const uint8_t *)ctx->perm.p;
    spec.args.win = P2Z_SORT_WINDOW;
  }
  auto launch_sort = [&](cudaStream_t s) {
    const int64_t nwin = (s1 - s0 + P2Z_SORT_WINDOW - 1) / P2Z_SORT_WINDOW;
    k_sort_windows<<<(unsigned)nwin, P2Z_SORT_WINDOW, 0, s>>>(base.mask, (uint8_t *)ctx->perm.p, s0, s1,
                                                               P2Z_SORT_WINDOW, all_layers(pl.nlayer));
    return cudaGetLastError();
  };
  if (schedule == P2Z_SCHED_FLAT) {
    if (sort) P2Z_CUDA(ctx, launch_sort(st));
    spec.kind = KIND_FLAT;
    P2Z_CUDA(ctx, dispatch(spec, st));
    ++*launches;
    return P2Z_OK;
  }
  // persistent (staged or not)
  spec.kind = schedule == P2Z_SCHED_STAGED ? KIND_STAGED : KIND_PERSISTENT;
  if (spec.kind == KIND_STAGED &&
      (pl.B != 32 || pl.soa || (((uintptr_t)base.trk | (uintptr_t)base.hits) & 15u) != 0 || s0 % 32 || s1 % 32))
    return fail(ctx, P2Z_UNSUPPORTED, "the staged schedule needs bsize 32, the AOSOA layout and 16-byte aligned "
                                      "track and hit arrays");
  const int occ = occupancy(spec);
  if (occ <= 0) return fail(ctx, P2Z_CUDA_ERROR, "occupancy query failed for the persistent kernel");
  const int64_t items = (s1 - s0 + 32 / spec.tpt - 1) / (32 / spec.tpt);
  const int64_t warps_per_cta = spec.block / 32;
  spec.grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)occ * ctx->num_sms, (items + warps_per_cta - 1) / warps_per_cta));
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  P2Z_CUDA(ctx, cudaStreamIsCapturing(st, &cap));
  const bool use_graph = !(pl.flags & P2Z_FLAG_NO_GRAPH) && cap == cudaStreamCaptureStatusNone;
  if (!use_graph) {
    if (sort) P2Z_CUDA(ctx, launch_sort(st));
    P2Z_CUDA(ctx, cudaMemsetAsync(queue, 0, sizeof(unsigned long long), st));
    P2Z_CUDA(ctx, dispatch(spec, st));
    ++*launches;
    return P2Z_OK;
  }
  GraphKey key;
  std::memset(&key, 0, sizeof key);
  key.args = spec.args;
  key.bsize = spec.bsize;
  key.upd = spec.upd;
  key.sc = spec.sc;
  key.block = spec.block;
  key.grid = spec.grid;
  key.masked = spec.masked;
  key.soa = spec.soa;
  key.kind = spec.kind;
  key.tpt = spec.tpt;
  if (!(ctx->has_graph && ctx->gkey == key)) {
    if (ctx->gexec) {
      cudaGraphExecDestroy(ctx->gexec);
      ctx->gexec = nullptr;
    }
    ctx->has_graph = false;
    // The graph is recorded on the context's own stream, which can always be
    // captured (the caller's may be the legacy default stream, which cannot),
    // and replayed on the caller's stream below.
    cudaGraph_t g = nullptr;
    cudaStream_t cs = ctx->stream;
    P2Z_CUDA(ctx, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    cudaError_t e0 = sort ? launch_sort(cs) : cudaSuccess;
    cudaError_t e1 = cudaMemsetAsync(queue, 0, sizeof(unsigned long long), cs);
    if (e1 == cudaSuccess) e1 = e0;
    cudaError_t e2 = dispatch(spec, cs);
    cudaError_t e3 = cudaStreamEndCapture(cs, &g);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      return fail(ctx, P2Z_CUDA_ERROR, "graph capture of the persistent launch failed: %s / %s / %s",
                  cudaGetErrorString(e1), cudaGetErrorString(e2), cudaGetErrorString(e3));
    }
    cudaError_t e4 = cudaGraphInstantiate(&ctx->gexec, g, 0);
    cudaGraphDestroy(g);
    if (e4 != cudaSuccess) return fail(ctx, P2Z_CUDA_ERROR, "cudaGraphInstantiate: %s", cudaGetErrorString(e4));
    ctx->gkey = key;
    ctx->has_graph = true;
  }
  P2Z_CUDA(ctx, cudaGraphLaunch(ctx->gexec, st));
  ++*launches;
  return P2Z_OK;
}

// Applies the autotuner's measurement for this kind of run to the fields the
// caller left open (block_threads = 0, schedule = AUTO -- with the window
// sorting measured with that schedule --, threads_per_track = 0), then
// resolves AUTO.  A tuned shape whose schedule the caller overrides
// with STAGED keeps one thread per track.
int resolve_schedule(p2z_context *ctx, Plan &pl, const p2z_config *cfg, bool masked) {
  masked = masked || pl.uneven;
  if (ctx) {
    for (const Tuned &t : ctx->tuned) {
      if (t.upd == pl.upd && t.sc == pl.sc && t.B == pl.B && t.soa == pl.soa && t.masked == masked) {
        if (cfg->block_threads == 0) pl.block = t.block;
        if (pl.schedule == P2Z_SCHED_AUTO) {
          pl.schedule = t.schedule;
          if (t.sort) pl.flags |= P2Z_FLAG_SORT_WINDOWS;
        }
        if (cfg->threads_per_track == 0 && pl.schedule != P2Z_SCHED_STAGED) pl.tpt = t.tpt;
        break;
      }
    }
  }
  if (pl.schedule != P2Z_SCHED_AUTO) return pl.schedule;
  return masked ? P2Z_SCHED_PERSISTENT : P2Z_SCHED_FLAT;
}

// Hit words an update kind reads per present layer: the 2-D updates the first
// 6 (x, y, z, V00, V10, V11), the 3-D ones all 9.
int hit_words_read(int upd) { return (upd == UPDK_3X3_F64 || upd == UPDK_3X3_COMP) ? 9 : 6; }

// P2Z_FLAG_CHECK_INPUTS: the scan of slots [s0, s1) on st (status bit 2).
p2z_status enqueue_check(p2z_context *ctx, const Plan &pl, const RunArgs &base, int64_t s0, int64_t s1,
                         cudaStream_t st) {
  RunArgs a = base;
  a.slot_begin = s0;
  a.slot_end = s1;
  a.ws = pl.nslots;
  P2Z_CUDA(ctx, launch_check_inputs(a, pl.soa ? 0 : pl.B, hit_words_read(pl.upd), st));
  return P2Z_OK;
}

// Real lanes per batch of uneven events (built only where the padding mask
// needs it: one byte per batch).
std::vector<uint8_t> batch_valid(const Plan &pl) {
  std::vector<uint8_t> v;
  v.reserve((size_t)pl.nbatches);
  const int64_t nev = (int64_t)pl.ev_slot_begin.size() - 1;
  for (int64_t e = 0; e < nev; ++e) {
    const int64_t n = pl.event_ntrks[e];
    for (int64_t left = n; left > 0; left -= pl.B) v.push_back((uint8_t)(left >= pl.B ? pl.B : left));
  }
  return v;
}

// Builds the padding mask of uneven events into ctx->valid / ctx->mask.
p2z_status internal_mask(p2z_context *ctx, const Plan &pl, cudaStream_t st, const uint32_t **out) {
  p2z_status r = ensure(ctx, ctx->mask, sizeof(uint32_t) * (size_t)pl.nslots);
  if (r != P2Z_OK) return r;
  *out = (const uint32_t *)ctx->mask.p;
  if (pl.nslots == 0) return P2Z_OK;
  // the mask depends on the batch width, the layers and the events' track counts only: a call with
  // the same ones as the last build reuses it (calls on one context are ordered, see p2z.h)
  const int64_t nev = (int64_t)pl.ev_slot_begin.size() - 1;
  std::vector<int64_t> key = {(int64_t)(uintptr_t)ctx->mask.p, pl.B, pl.nlayer};
  key.insert(key.end(), pl.event_ntrks, pl.event_ntrks + nev);
  if (key == ctx->mask_key) return P2Z_OK;
  ctx->mask_key.clear();
  const std::vector<uint8_t> valid = batch_valid(pl);
  r = ensure(ctx, ctx->valid, valid.size());
  if (r != P2Z_OK) return r;
  // (pageable source: the copy is staged before the call returns)
  P2Z_CUDA(ctx, cudaMemcpyAsync(ctx->valid.p, valid.data(), valid.size(), cudaMemcpyHostToDevice, st));
  k_fill_mask<<<(unsigned)((pl.nslots + 255) / 256), 256, 0, st>>>((uint32_t *)ctx->mask.p, (const uint8_t *)ctx->valid.p,
                                                                   pl.nslots, pl.B, all_layers(pl.nlayer));
  P2Z_CUDA(ctx, cudaGetLastError());
  ctx->mask_key = std::move(key);
  return P2Z_OK;
}

p2z_status count_updates(p2z_context *ctx, const Plan &pl, const uint32_t *d_mask, cudaStream_t st, int64_t *out) {
  if (!d_mask) {
    *out = pl.nslots * pl.nlayer;
    return P2Z_OK;
  }
  if (pl.nslots == 0) {
    *out = 0;
    return P2Z_OK;
  }
  unsigned long long *d = ctx->d_queue + 2;  // scratch word
  P2Z_CUDA(ctx, cudaMemsetAsync(d, 0, sizeof(unsigned long long), st));
  k_count_updates<<<ctx->num_sms * 4, 256, 0, st>>>(d_mask, pl.nslots, all_layers(pl.nlayer), d);
  P2Z_CUDA(ctx, cudaGetLastError());
  unsigned long long h = 0;
  P2Z_CUDA(ctx, cudaMemcpyAsync(&h, d, sizeof h, cudaMemcpyDeviceToHost, st));
  P2Z_CUDA(ctx, cudaStreamSynchronize(st));
  *out = (int64_t)h;
  return P2Z_OK;
}

// p2z_run, SoA layout: host->device copy of slots [s0, s0 + n) of every
// element row of the tracks (28 rows) and hits (nlayer x 9 rows, or the first
// 6 of each layer's 9 when `six`), with pitched copies.
p2z_status copy_soa_chunk(p2z_context *ctx, const Plan &pl, const void *trk_in, const void *hits, int64_t s0, int64_t n,
                          bool six, cudaStream_t st, int64_t *h2d) {
  const size_t pitch = (size_t)pl.nslots * 4, off = (size_t)s0 * 4, w = (size_t)n * 4;
  P2Z_CUDA(ctx, cudaMemcpy2DAsync((char *)ctx->trk.p + off, pitch, (const char *)trk_in + off, pitch, w, TRK_WORDS,
                                  cudaMemcpyHostToDevice, st));
  *h2d += (int64_t)(w * TRK_WORDS);
  if (!six) {
    P2Z_CUDA(ctx, cudaMemcpy2DAsync((char *)ctx->hits.p + off, pitch, (const char *)hits + off, pitch, w,
                                    (size_t)HIT_WORDS * pl.nlayer, cudaMemcpyHostToDevice, st));
    *h2d += (int64_t)(w * HIT_WORDS * pl.nlayer);
    return P2Z_OK;
  }
  // rows (l, e) for e < 6 of each layer: a 3-D box of the [nlayer][9][nslots] array
  cudaMemcpy3DParms c;
  std::memset(&c, 0, sizeof c);
  c.srcPtr = make_cudaPitchedPtr(const_cast<void *>(hits), pitch, pitch, HIT_WORDS);
  c.dstPtr = make_cudaPitchedPtr(ctx->hits.p, pitch, pitch, HIT_WORDS);
  c.srcPos = make_cudaPos(off, 0, 0);
  c.dstPos = make_cudaPos(off, 0, 0);
  c.extent = make_cudaExtent(w, 6, (size_t)pl.nlayer);
  c.kind = cudaMemcpyHostToDevice;
  P2Z_CUDA(ctx, cudaMemcpy3DAsync(&c, st));
  *h2d += (int64_t)(w * 6 * pl.nlayer);
  return P2Z_OK;
}

}  // namespace

namespace p2z {
// Records the message p2z_last_error(NULL) returns (failures with no context).
void set_context_free_error(const char *msg) { fail(nullptr, P2Z_OK, "%s", msg); }

// Autotuner hooks: the context's device and stream, its error message, and
// the record of a measured best launch shape for the runs cfg describes.
int context_device(const p2z_context *ctx) { return ctx->device; }
cudaStream_t context_stream(const p2z_context *ctx) { return ctx->stream; }
p2z_status context_fail(p2z_context *ctx, p2z_status st, const char *msg) { return fail(ctx, st, "%s", msg); }
// Device scratch owned by the context, at least `bytes` long (nullptr on failure).
void *context_scratch(p2z_context *ctx, size_t bytes) {
  return ensure(ctx, ctx->aux, bytes) == P2Z_OK ? ctx->aux.p : nullptr;
}
p2z_status record_tuned(p2z_context *ctx, const p2z_config *cfg, bool masked, int block, int schedule, int tpt,
                        bool sort) {
  Plan pl;
  p2z_status r = make_plan(ctx, cfg, pl);
  if (r != P2Z_OK) return r;
  Tuned t{pl.upd, pl.sc, pl.B, pl.soa, masked || pl.uneven, block, schedule, tpt, sort};
  for (Tuned &o : ctx->tuned) {
    if (o.upd == t.upd && o.sc == t.sc && o.B == t.B && o.soa == t.soa && o.masked == t.masked) {
      o = t;
      return P2Z_OK;
    }
  }
  ctx->tuned.push_back(t);
  return P2Z_OK;
}
}  // namespace p2z

extern "C" {

p2z_status p2z_config_init(p2z_config *cfg, int32_t bsize, int64_t nevts, int64_t ntrks, int32_t nlayer) {
  if (!cfg) return fail(nullptr, P2Z_BAD_ARG, "config is NULL");
  std::memset(cfg, 0, sizeof *cfg);
  cfg->abi_version = P2Z_ABI_VERSION;
  cfg->bsize = bsize;
  cfg->nevts = nevts;
  cfg->ntrks = ntrks;
  cfg->nlayer = nlayer;
  cfg->niter = 1;
  cfg->update = P2Z_UPDATE_V2;
  return P2Z_OK;
}

const char *p2z_status_string(p2z_status s) {
  switch (s) {
    case P2Z_OK: return "ok";
    case P2Z_BAD_ARG: return "bad argument";
    case P2Z_OOM: return "out of memory";
    case P2Z_NONFINITE_INPUT: return "non-finite input";
    case P2Z_SINGULAR: return "singular residual covariance";
    case P2Z_TIMEOUT: return "timeout";
    case P2Z_CUDA_ERROR: return "CUDA error";
    case P2Z_NO_DEVICE: return "no CUDA device";
    case P2Z_UNSUPPORTED: return "unsupported";
    case P2Z_NOT_READY: return "not ready";
  }
  return "unknown status";
}

const char *p2z_last_error(const p2z_context *ctx) {
  if (ctx) return ctx->last_error.c_str();
  std::lock_guard<std::mutex> lk(g_err_mu);
  return g_last_error.c_str();
}

int p2z_version(char *buf, size_t buflen) {
  if (buf && buflen) {
    std::snprintf(buf, buflen, "libp2z abi %d, sm_100a, built %s %s, CUDA %d", P2Z_ABI_VERSION, __DATE__, __TIME__,
                  CUDART_VERSION);
  }
  return P2Z_ABI_VERSION;
}

size_t p2z_sizeof_mptrk(int bsize) { return valid_bsize(bsize) ? (size_t)TRK_WORDS * bsize * 4 : 0; }
size_t p2z_sizeof_mphit(int bsize) { return valid_bsize(bsize) ? (size_t)HIT_WORDS * bsize * 4 : 0; }

int64_t p2z_num_batches(const p2z_config *cfg) {
  Plan pl;
  if (make_plan(nullptr, cfg, pl) != P2Z_OK) return -1;
  return pl.nbatches;
}

p2z_status p2z_create(int device, p2z_context **out) {
  if (!out) return fail(nullptr, P2Z_BAD_ARG, "out is NULL");
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(nullptr, P2Z_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(e));
  }
  if (device < 0) {
    if (cudaGetDevice(&device) != cudaSuccess) return fail(nullptr, P2Z_NO_DEVICE, "cudaGetDevice failed");
  }
  if (device >= ndev) return fail(nullptr, P2Z_BAD_ARG, "device %d >= device count %d", device, ndev);
  p2z_context *c = new p2z_context();
  c->device = device;
  auto bail = [&](const char *what, cudaError_t err) {
    std::string msg = std::string(what) + ": " + cudaGetErrorString(err);
    p2z_destroy(c);
    return fail(nullptr, err == cudaErrorMemoryAllocation ? P2Z_OOM : P2Z_CUDA_ERROR, "%s", msg.c_str());
  };
  if ((e = cudaSetDevice(device)) != cudaSuccess) return bail("cudaSetDevice", e);
  if ((e = cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess)
    return bail("cudaDeviceGetAttribute", e);
  if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) return bail("stream", e);
  for (int i = 0; i < 2; ++i) {
    if ((e = cudaStreamCreateWithFlags(&c->copy[i], cudaStreamNonBlocking)) != cudaSuccess) return bail("stream", e);
    if ((e = cudaEventCreateWithFlags(&c->join[i], cudaEventDisableTiming)) != cudaSuccess) return bail("event", e);
  }
  if ((e = cudaEventCreate(&c->ev0)) != cudaSuccess) return bail("event", e);
  if ((e = cudaEventCreate(&c->ev1)) != cudaSuccess) return bail("event", e);
  if ((e = cudaEventCreate(&c->ev2)) != cudaSuccess) return bail("event", e);
  if ((e = cudaEventCreate(&c->ev3)) != cudaSuccess) return bail("event", e);
  if ((e = cudaMalloc(&c->d_status, sizeof(unsigned int))) != cudaSuccess) return bail("cudaMalloc status", e);
  if ((e = cudaMalloc(&c->d_queue, 4 * sizeof(unsigned long long))) != cudaSuccess) return bail("cudaMalloc queue", e);
  if ((e = cudaMemset(c->d_status, 0, sizeof(unsigned int))) != cudaSuccess) return bail("cudaMemset", e);
  if ((e = cudaHostAlloc(&c->h_status, sizeof(unsigned int), cudaHostAllocDefault)) != cudaSuccess)
    return bail("cudaHostAlloc status", e);
  *out = c;
  return P2Z_OK;
}

p2z_status p2z_destroy(p2z_context *c) {
  if (!c) return P2Z_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (int i = 0; i < 2; ++i)
    if (c->copy[i]) cudaStreamSynchronize(c->copy[i]);
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  if (c->run_exec) cudaGraphExecDestroy(c->run_exec);
  for (DevBuf *b : {&c->trk, &c->hits, &c->out, &c->mask, &c->valid, &c->aux, &c->perm})
    if (b->p) cudaFree(b->p);
  if (c->d_status) cudaFree(c->d_status);
  if (c->h_status) cudaFreeHost(c->h_status);
  if (c->d_queue) cudaFree(c->d_queue);
  for (cudaEvent_t ev : {c->ev0, c->ev1, c->ev2, c->ev3, c->join[0], c->join[1], c->ev_fork})
    if (ev) cudaEventDestroy(ev);
  for (int i = 0; i < kEventStreams; ++i) {
    if (c->ev_streams[i]) {
      cudaStreamSynchronize(c->ev_streams[i]);
      cudaStreamDestroy(c->ev_streams[i]);
    }
    if (c->ev_join[i]) cudaEventDestroy(c->ev_join[i]);
  }
  for (int i = 0; i < 2; ++i)
    if (c->copy[i]) cudaStreamDestroy(c->copy[i]);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return P2Z_OK;
}

p2z_status p2z_run_device(p2z_context *ctx, const p2z_config *cfg, const void *d_trk_in, const void *d_hits,
                          const uint32_t *d_hit_mask, void *d_trk_out, void *stream, p2z_stats *stats) {
  if (!ctx) return fail(nullptr, P2Z_BAD_ARG, "context is NULL");
  Plan pl;
  p2z_status r = make_plan(ctx, cfg, pl);
  if (r != P2Z_OK) return r;
  if (pl.nslots > 0 && (!d_trk_in || !d_hits || !d_trk_out)) return fail(ctx, P2Z_BAD_ARG, "NULL device buffer");
  if (d_trk_in == d_trk_out && pl.nslots > 0) return fail(ctx, P2Z_BAD_ARG, "d_trk_out must not alias d_trk_in");
  P2Z_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  const uint32_t *mask = d_hit_mask;
  if (!mask && pl.uneven) {
    r = internal_mask(ctx, pl, st, &mask);
    if (r != P2Z_OK) return r;
  }
  RunArgs base;
  std::memset(&base, 0, sizeof base);
  base.trk = (const float *)d_trk_in;
  base.hits = (const float *)d_hits;
  base.out = (float *)d_trk_out;
  base.mask = mask;
  base.nlayer = pl.nlayer;
  base.kfact = pl.kfact;
  base.status = ctx->d_status;
  const int schedule = resolve_schedule(ctx, pl, cfg, mask != nullptr);
  int launches = 0;
  if ((pl.flags & P2Z_FLAG_CHECK_INPUTS) && pl.nslots > 0) {
    // synchronous: the pass runs only on finite inputs
    P2Z_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(unsigned int), st));
    r = enqueue_check(ctx, pl, base, 0, pl.nslots, st);
    if (r != P2Z_OK) return r;
    P2Z_CUDA(ctx, cudaMemcpyAsync(ctx->h_status, ctx->d_status, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
    P2Z_CUDA(ctx, cudaStreamSynchronize(st));
    if (*(volatile unsigned int *)ctx->h_status & 4u)
      return fail(ctx, P2Z_NONFINITE_INPUT, "a track or hit word the pass reads is NaN or Inf");
  }
  // the status word is read back for stats and, without them, for P2Z_FLAG_STRICT (the call then
  // synchronises)
  const bool strict_only = !stats && (pl.flags & P2Z_FLAG_STRICT) && pl.nslots > 0;
  if (stats || strict_only) P2Z_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(unsigned int), st));
  if (stats) P2Z_CUDA(ctx, cudaEventRecord(ctx->ev0, st));
  for (int it = 0; it < pl.niter; ++it) {
    r = enqueue_pass(ctx, pl, base, 0, pl.nslots, schedule, st, ctx->d_queue, &launches);
    if (r != P2Z_OK) return r;
  }
  if (stats) {
    P2Z_CUDA(ctx, cudaEventRecord(ctx->ev1, st));
    P2Z_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
    float ms = 0.f;
    P2Z_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    unsigned int status = 0;
    P2Z_CUDA(ctx, cudaMemcpy(&status, ctx->d_status, sizeof status, cudaMemcpyDeviceToHost));
    std::memset(stats, 0, sizeof *stats);
    stats->kernel_ms = ms;
    stats->total_ms = ms;
    stats->track_slots = pl.nslots;
    r = count_updates(ctx, pl, mask, st, &stats->updates);
    if (r != P2Z_OK) return r;
    stats->launches = launches;
    stats->singular = (status & 1u) ? 1 : 0;
    if (status & 2u) return fail(ctx, P2Z_TIMEOUT, "a staged kernel's wait for a bulk copy ran out");
    if ((pl.flags & P2Z_FLAG_STRICT) && stats->singular)
      return fail(ctx, P2Z_SINGULAR, "a residual covariance with det <= 0 was met");
  } else if (strict_only) {
    P2Z_CUDA(ctx, cudaMemcpyAsync(ctx->h_status, ctx->d_status, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
    P2Z_CUDA(ctx, cudaStreamSynchronize(st));
    const unsigned int status = *(volatile unsigned int *)ctx->h_status;
    if (status & 2u) return fail(ctx, P2Z_TIMEOUT, "a staged kernel's wait for a bulk copy ran out");
    if (status & 1u) return fail(ctx, P2Z_SINGULAR, "a residual covariance with det <= 0 was met");
  } else {
    P2Z_CUDA(ctx, cudaGetLastError());
  }
  return P2Z_OK;
}

p2z_status p2z_run(p2z_context *ctx, const p2z_config *cfg, const void *trk_in, const void *hits,
                   const uint32_t *hit_mask, void *trk_out, p2z_stats *stats) {
  if (!ctx) return fail(nullptr, P2Z_BAD_ARG, "context is NULL");
  Plan pl;
  p2z_status r = make_plan(ctx, cfg, pl);
  if (r != P2Z_OK) return r;
  if (pl.nslots > 0 && (!trk_in || !hits || !trk_out)) return fail(ctx, P2Z_BAD_ARG, "NULL host buffer");
  P2Z_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t tb = p2z_sizeof_mptrk(pl.B), hb = p2z_sizeof_mphit(pl.B);
  const size_t trk_bytes = tb * (size_t)pl.nbatches;
  const size_t hit_bytes = hb * (size_t)pl.nbatches * pl.nlayer;
  if ((r = ensure(ctx, ctx->trk, trk_bytes)) != P2Z_OK) return r;
  if ((r = ensure(ctx, ctx->hits, hit_bytes)) != P2Z_OK) return r;
  if ((r = ensure(ctx, ctx->out, trk_bytes)) != P2Z_OK) return r;
  const bool user_mask = hit_mask != nullptr;
  const uint32_t *d_mask = nullptr;
  if (user_mask) {
    // ctx->mask is also the internal padding mask; a user mask replaces it.
    if ((r = ensure(ctx, ctx->mask, sizeof(uint32_t) * (size_t)pl.nslots)) != P2Z_OK) return r;
    ctx->mask_key.clear();
    d_mask = (const uint32_t *)ctx->mask.p;
  }
  cudaStream_t s0 = ctx->copy[0], s1 = ctx->copy[1];
  if (!user_mask && pl.uneven) {
    r = internal_mask(ctx, pl, s0, &d_mask);
    if (r != P2Z_OK) return r;
    P2Z_CUDA(ctx, cudaEventRecord(ctx->join[0], s0));
    P2Z_CUDA(ctx, cudaStreamWaitEvent(s1, ctx->join[0], 0));
  }
  RunArgs base;
  std::memset(&base, 0, sizeof base);
  base.trk = (const float *)ctx->trk.p;
  base.hits = (const float *)ctx->hits.p;
  base.out = (float *)ctx->out.p;
  base.mask = d_mask;
  base.nlayer = pl.nlayer;
  base.kfact = pl.kfact;
  base.status = ctx->d_status;
  int schedule = resolve_schedule(ctx, pl, cfg, d_mask != nullptr);
  // The per-event form is timed as it stands: copies first, then one launch per event.
  const bool per_event = schedule == P2Z_SCHED_PER_EVENT;
  // Only the 2-D updates read just the first 6 of the 9 hit words.
  const bool six = (pl.upd == UPDK_V2 || pl.upd == UPDK_V2_COMP || pl.upd == UPDK_F64 || pl.upd == UPDK_V2_REF) &&
                   !(pl.flags & P2Z_FLAG_FULL_HITS);
  const int64_t nchunk = per_event ? 1 : std::max<int64_t>(1, std::min<int64_t>(P2Z_RUN_MAX_CHUNKS, pl.nbatches / 64));
  const int64_t cb = nchunk ? (pl.nbatches + nchunk - 1) / nchunk : 0;
  int launches = 0;
  int64_t h2d = 0, d2h = 0;
  // P2Z_FLAG_CHECK_INPUTS: each chunk is scanned after its copies, before its pass
  const bool check = (pl.flags & P2Z_FLAG_CHECK_INPUTS) != 0;
  // The work of one call on the two copy streams: the status reset, then per
  // chunk the host->device copies, the pass and the device->host copy,
  // alternating between s0 and s1 (s1 forks from and joins back into s0).
  auto pipeline = [&]() -> p2z_status {
    P2Z_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(unsigned int), s0));
    P2Z_CUDA(ctx, cudaEventRecord(ctx->join[0], s0));
    P2Z_CUDA(ctx, cudaStreamWaitEvent(s1, ctx->join[0], 0));
    for (int it = 0; it < pl.niter; ++it) {
      for (int64_t c = 0; c < nchunk; ++c) {
        cudaStream_t st = (c & 1) ? s1 : s0;
        const int64_t b0 = c * cb, b1 = std::min(pl.nbatches, b0 + cb);
        if (b1 <= b0) continue;
        const int64_t nbc = b1 - b0;
        if (pl.soa) {
          // slots [b0*B, b1*B) of every element row: pitched copies
          r = copy_soa_chunk(ctx, pl, trk_in, hits, b0 * pl.B, nbc * pl.B, six, st, &h2d);
          if (r != P2Z_OK) return r;
        } else {
          P2Z_CUDA(ctx, cudaMemcpyAsync((char *)ctx->trk.p + b0 * tb, (const char *)trk_in + b0 * tb, nbc * tb,
                                        cudaMemcpyHostToDevice, st));
          h2d += nbc * tb;
          const size_t hrow = hb, hrows = (size_t)nbc * pl.nlayer;
          const size_t hoff = (size_t)b0 * pl.nlayer * hb;
          if (six) {
            const size_t w = 6 * (size_t)pl.B * 4;
            P2Z_CUDA(ctx, cudaMemcpy2DAsync((char *)ctx->hits.p + hoff, hrow, (const char *)hits + hoff, hrow, w, hrows,
                                            cudaMemcpyHostToDevice, st));
            h2d += (int64_t)(w * hrows);
          } else {
            P2Z_CUDA(ctx, cudaMemcpyAsync((char *)ctx->hits.p + hoff, (const char *)hits + hoff, hrow * hrows,
                                          cudaMemcpyHostToDevice, st));
            h2d += (int64_t)(hrow * hrows);
          }
        }
        if (user_mask) {
          P2Z_CUDA(ctx, cudaMemcpyAsync((char *)ctx->mask.p + b0 * pl.B * 4, (const char *)hit_mask + b0 * pl.B * 4,
                                        nbc * pl.B * 4, cudaMemcpyHostToDevice, st));
          h2d += nbc * pl.B * 4;
        }
        if (check) {
          r = enqueue_check(ctx, pl, base, b0 * pl.B, b1 * pl.B, st);
          if (r != P2Z_OK) return r;
        }
        if (!per_event) {
          r = enqueue_pass(ctx, pl, base, b0 * pl.B, b1 * pl.B,
                           (schedule == P2Z_SCHED_PERSISTENT || schedule == P2Z_SCHED_STAGED) ? P2Z_SCHED_FLAT : schedule,
                           st, ctx->d_queue + (c & 1), &launches);
          if (r != P2Z_OK) return r;
          if (pl.soa) {
            const size_t pitch = (size_t)pl.nslots * 4, off = (size_t)b0 * pl.B * 4, w = (size_t)nbc * pl.B * 4;
            P2Z_CUDA(ctx, cudaMemcpy2DAsync((char *)trk_out + off, pitch, (const char *)ctx->out.p + off, pitch, w,
                                            TRK_WORDS, cudaMemcpyDeviceToHost, st));
          } else {
            P2Z_CUDA(ctx, cudaMemcpyAsync((char *)trk_out + b0 * tb, (const char *)ctx->out.p + b0 * tb, nbc * tb,
                                          cudaMemcpyDeviceToHost, st));
          }
          d2h += nbc * tb;
        }
      }
      if (per_event) {
        r = enqueue_pass(ctx, pl, base, 0, pl.nslots, P2Z_SCHED_PER_EVENT, s0, ctx->d_queue, &launches);
        if (r != P2Z_OK) return r;
        P2Z_CUDA(ctx, cudaMemcpyAsync(trk_out, ctx->out.p, trk_bytes, cudaMemcpyDeviceToHost, s0));
        d2h += trk_bytes;
      }
    }
    P2Z_CUDA(ctx, cudaEventRecord(ctx->join[1], s1));
    P2Z_CUDA(ctx, cudaStreamWaitEvent(s0, ctx->join[1], 0));
    P2Z_CUDA(ctx, cudaMemcpyAsync(ctx->h_status, ctx->d_status, sizeof(unsigned int), cudaMemcpyDeviceToHost, s0));
    return P2Z_OK;
  };
  // With page-locked host buffers a pipeline of at least kRunGraphMinChunks
  // passes over chunks (or per-event launches; niter passes each) is recorded once as a CUDA graph and
  // replayed while the plan and every buffer it touches stay the same: a call
  // then costs one graph launch instead of enqueueing each copy and kernel (up
  // to 16 chunks x 4-5 operations, or one launch per event).  A shorter
  // pipeline is enqueued directly: its first copy then starts while the rest
  // is still being enqueued, which a graph launch does not allow (one B200,
  // one event from page-locked buffers: direct 3-6 us faster per call from
  // 256 to 4096 tracks, one and two chunks; the graph 1 us faster at 9600
  // tracks, four chunks).  Pageable buffers are copied through the driver's
  // staging path, which a graph cannot hold, so they take the direct path, as
  // does P2Z_FLAG_NO_GRAPH.
  constexpr int64_t kRunGraphMinChunks = 4;
  const int64_t pipeline_ops = (per_event ? (int64_t)pl.ev_slot_begin.size() - 1 : nchunk) * pl.niter;
  const bool graph = !(pl.flags & P2Z_FLAG_NO_GRAPH) && pl.nslots > 0 && pipeline_ops >= kRunGraphMinChunks &&
                     page_locked(trk_in) && page_locked(hits) && page_locked(trk_out) &&
                     (!user_mask || page_locked(hit_mask));
  if (graph) {
    // what enqueue_pass would allocate or create on first use, before recording
    if (d_mask && (pl.flags & P2Z_FLAG_SORT_WINDOWS) && (r = ensure(ctx, ctx->perm, (size_t)pl.nslots)) != P2Z_OK)
      return r;
    if (per_event && (pl.flags & P2Z_FLAG_PER_EVENT_STREAMS) && (r = event_streams(ctx)) != P2Z_OK) return r;
    int32_t kbits;
    std::memcpy(&kbits, &pl.kfact, sizeof kbits);
    std::vector<int64_t> key = {pl.B, pl.nlayer, pl.niter, kbits, pl.upd, pl.sc, pl.block, pl.tpt, (int64_t)pl.flags,
                                pl.nbatches, pl.soa, pl.uneven, schedule, user_mask,
                                (int64_t)(uintptr_t)trk_in, (int64_t)(uintptr_t)hits, (int64_t)(uintptr_t)hit_mask,
                                (int64_t)(uintptr_t)trk_out, (int64_t)(uintptr_t)ctx->trk.p,
                                (int64_t)(uintptr_t)ctx->hits.p, (int64_t)(uintptr_t)ctx->out.p,
                                (int64_t)(uintptr_t)ctx->mask.p, (int64_t)(uintptr_t)ctx->perm.p,
                                (int64_t)(uintptr_t)d_mask};
    key.insert(key.end(), pl.ev_slot_begin.begin(), pl.ev_slot_begin.end());
    if (!(ctx->run_exec && ctx->run_key == key)) {
      if (ctx->run_exec) cudaGraphExecDestroy(ctx->run_exec);
      ctx->run_exec = nullptr;
      ctx->run_key.clear();
      P2Z_CUDA(ctx, cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal));
      r = pipeline();
      cudaGraph_t g = nullptr;
      const cudaError_t e = cudaStreamEndCapture(s0, &g);
      if (r != P2Z_OK || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return r != P2Z_OK ? r : fail(ctx, P2Z_CUDA_ERROR, "recording p2z_run's pipeline: %s", cudaGetErrorString(e));
      }
      const cudaError_t e2 = cudaGraphInstantiate(&ctx->run_exec, g, 0);
      cudaGraphDestroy(g);
      if (e2 != cudaSuccess) {
        ctx->run_exec = nullptr;
        return fail(ctx, P2Z_CUDA_ERROR, "cudaGraphInstantiate: %s", cudaGetErrorString(e2));
      }
      ctx->run_key = std::move(key);
      ctx->run_launches = launches;
      ctx->run_h2d = h2d;
      ctx->run_d2h = d2h;
    }
    launches = ctx->run_launches;
    h2d = ctx->run_h2d;
    d2h = ctx->run_d2h;
    P2Z_CUDA(ctx, cudaEventRecord(ctx->ev0, s0));
    P2Z_CUDA(ctx, cudaGraphLaunch(ctx->run_exec, s0));
  } else {
    P2Z_CUDA(ctx, cudaEventRecord(ctx->ev0, s0));
    if ((r = pipeline()) != P2Z_OK) return r;
  }
  P2Z_CUDA(ctx, cudaEventRecord(ctx->ev1, s0));
  P2Z_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
  const unsigned int status = *(volatile unsigned int *)ctx->h_status;  // copied by the pipeline's last step
  if (stats) {
    float ms = 0.f;
    P2Z_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    std::memset(stats, 0, sizeof *stats);
    stats->total_ms = ms;
    stats->track_slots = pl.nslots;
    stats->h2d_bytes = h2d;
    stats->d2h_bytes = d2h;
    stats->launches = launches;
    stats->singular = (status & 1u) ? 1 : 0;
    r = count_updates(ctx, pl, d_mask, s0, &stats->updates);
    if (r != P2Z_OK) return r;
  }
  if (status & 4u) return fail(ctx, P2Z_NONFINITE_INPUT, "a track or hit word the pass read is NaN or Inf");
  if ((pl.flags & P2Z_FLAG_STRICT) && (status & 1u))
    return fail(ctx, P2Z_SINGULAR, "a residual covariance with det <= 0 was met");
  return P2Z_OK;
}

p2z_status p2z_step_device(p2z_context *ctx, int bsize, int64_t nbatches, void *d_trk, const void *d_hits, int nlayer,
                           int layer, int what, int update, float kfact) {
  if (!ctx) return fail(nullptr, P2Z_BAD_ARG, "context is NULL");
  if (!valid_bsize(bsize)) return fail(ctx, P2Z_UNSUPPORTED, "bsize %d not in {8,16,32,64}", bsize);
  if (nbatches < 0 || nlayer < 1 || layer < 0 || layer >= nlayer || what < 1 || what > 3)
    return fail(ctx, P2Z_BAD_ARG, "bad step arguments");
  if (update != P2Z_UPDATE_V2) return fail(ctx, P2Z_UNSUPPORTED, "p2z_step_device implements the V2 update only");
  if (nbatches > 0 && (!d_trk || !d_hits)) return fail(ctx, P2Z_BAD_ARG, "NULL device buffer");
  P2Z_CUDA(ctx, cudaSetDevice(ctx->device));
  const float kf = kfact != 0.f ? kfact : (float)(100. / (-0.299792458 * 3.8112));
  P2Z_CUDA(ctx, launch_step(bsize, (float *)d_trk, (const float *)d_hits, nbatches * bsize, nlayer, layer, what, kf,
                            ctx->stream));
  P2Z_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return P2Z_OK;
}

p2z_status p2z_host_alloc(void **ptr, size_t bytes) {
  if (!ptr) return fail(nullptr, P2Z_BAD_ARG, "ptr is NULL");
  cudaError_t e = cudaHostAlloc(ptr, bytes ? bytes : 1, cudaHostAllocPortable);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *ptr = nullptr;
    return fail(nullptr, e == cudaErrorMemoryAllocation ? P2Z_OOM : P2Z_CUDA_ERROR, "cudaHostAlloc(%zu): %s", bytes,
                cudaGetErrorString(e));
  }
  return P2Z_OK;
}

p2z_status p2z_device_alloc(p2z_context *ctx, void **d_ptr, size_t bytes) {
  if (!ctx || !d_ptr) return fail(ctx, P2Z_BAD_ARG, "context or pointer is NULL");
  *d_ptr = nullptr;
  P2Z_CUDA(ctx, cudaSetDevice(ctx->device));
  P2Z_CUDA(ctx, cudaMalloc(d_ptr, bytes ? bytes : 1));
  return P2Z_OK;
}

p2z_status p2z_device_free(p2z_context *ctx, void *d_ptr) {
  if (!ctx) return fail(nullptr, P2Z_BAD_ARG, "context is NULL");
  if (!d_ptr) return P2Z_OK;
  P2Z_CUDA(ctx, cudaSetDevice(ctx->device));
  P2Z_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  P2Z_CUDA(ctx, cudaFree(d_ptr));
  return P2Z_OK;
}

p2z_status p2z_copy(p2z_context *ctx, void *dst, const void *src, size_t bytes) {
  if (!ctx) return fail(nullptr, P2Z_BAD_ARG, "context is NULL");
  if (bytes == 0) return P2Z_OK;
  if (!dst || !src) return fail(ctx, P2Z_BAD_ARG, "NULL copy pointer");
  P2Z_CUDA(ctx, cudaSetDevice(ctx->device));
  P2Z_CUDA(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, ctx->stream));
  P2Z_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return P2Z_OK;
}

p2z_status p2z_host_free(void *ptr) {
  if (!ptr) return P2Z_OK;
  cudaError_t e = cudaFreeHost(ptr);
  if (e != cudaSuccess) return fail(nullptr, P2Z_CUDA_ERROR, "cudaFreeHost: %s", cudaGetErrorString(e));
  return P2Z_OK;
}

}  // extern "C"
