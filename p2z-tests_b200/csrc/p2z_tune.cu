// p2z_tune.cu -- layout conversion between bsizes / AOSOA / SoA on the device,
// and the autotuner that measures every (bsize, layout, schedule, block size,
// threads per track) on the caller's data.  Neither has a counterpart in the reference, whose
// bsize is a compile-time macro (src/propagate-toz-test_OMP.cpp:22-24) and
// whose launch shape is fixed per build (src/propagate-toz-test_CUDA_v4.cu:
// 57-72).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "p2z.h"
#include "p2z_kernels.cuh"

namespace p2z {
void set_context_free_error(const char *msg);
int context_device(const p2z_context *ctx);
cudaStream_t context_stream(const p2z_context *ctx);
p2z_status context_fail(p2z_context *ctx, p2z_status st, const char *msg);
p2z_status record_tuned(p2z_context *ctx, const p2z_config *cfg, bool masked, int block, int schedule, int tpt,
                        bool sort);
}  // namespace p2z

using namespace p2z;

namespace {

// One side of a conversion: where slot s, row r lives.  Rows: tracks 0..27
// (element), hits l*9 + e, masks 0.
struct Side {
  int B;            // batch width (AOSOA)
  int soa;          // 1: SoA
  int64_t ns;       // slots in the array
  const int64_t *beg;  // device: first slot of each event (nevts + 1)
};

enum { ARR_TRK = 0, ARR_HIT = 1, ARR_MASK = 2 };

__device__ __forceinline__ int64_t word_index(const Side &d, int arr, int nlayer, int64_t s, int r) {
  if (arr == ARR_MASK) return s;
  if (d.soa) return (int64_t)r * d.ns + s;
  const int64_t b = s / d.B, t = s % d.B;
  if (arr == ARR_TRK) return b * (int64_t)(TRK_WORDS * d.B) + (int64_t)r * d.B + t;
  const int l = r / HIT_WORDS, e = r % HIT_WORDS;
  return (b * nlayer + l) * (int64_t)(HIT_WORDS * d.B) + (int64_t)e * d.B + t;
}

// Destination slot s (x), row (y): copy the word of the same track from the
// source, or 0 for a padding slot.  Words are moved as raw 32-bit patterns.
__global__ void k_relayout(const uint32_t *__restrict__ src, uint32_t *__restrict__ dst, Side from, Side to,
                           const int64_t *__restrict__ counts, int nevts, int arr, int nlayer) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= to.ns) return;
  const int r = blockIdx.y;
  // event of s: the last e with to.beg[e] <= s
  int lo = 0, hi = nevts - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (to.beg[mid] <= s) lo = mid;
    else hi = mid - 1;
  }
  const int64_t i = s - to.beg[lo];
  uint32_t v = 0u;
  if (i < counts[lo]) v = src[word_index(from, arr, nlayer, from.beg[lo] + i, r)];
  dst[word_index(to, arr, nlayer, s, r)] = v;
}

// Per-event track counts of a config (uniform or uneven).
bool event_counts(const p2z_config *c, std::vector<int64_t> &n) {
  n.assign((size_t)std::max<int64_t>(0, c->nevts), 0);
  for (int64_t e = 0; e < c->nevts; ++e) n[e] = c->event_ntrks ? c->event_ntrks[e] : c->ntrks;
  return true;
}

std::vector<int64_t> event_begins(const std::vector<int64_t> &n, int B) {
  std::vector<int64_t> beg(n.size() + 1, 0);
  for (size_t e = 0; e < n.size(); ++e) beg[e + 1] = beg[e] + (n[e] + B - 1) / B * B;
  return beg;
}

#define TUNE_CUDA(ctx, call)                                                                    \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) {                                                                    \
      char m_[300];                                                                             \
      std::snprintf(m_, sizeof m_, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                    __LINE__);                                                                  \
      return context_fail((ctx), e_ == cudaErrorMemoryAllocation ? P2Z_OOM : P2Z_CUDA_ERROR, m_); \
    }                                                                                           \
  } while (0)

// Device buffers freed on scope exit.
struct Scratch {
  std::vector<void *> p;
  ~Scratch() {
    for (void *q : p)
      if (q) cudaFree(q);
  }
  cudaError_t alloc(void **out, size_t bytes) {
    *out = nullptr;
    if (bytes == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(out, bytes);
    if (e == cudaSuccess) p.push_back(*out);
    return e;
  }
};

p2z_status relayout(p2z_context *ctx, const p2z_config *from, const p2z_config *to, const void *trk_in,
                    const void *hits_in, const uint32_t *mask_in, void *trk_out, void *hits_out, uint32_t *mask_out,
                    cudaStream_t st, Scratch &scr) {
  char msg[200];
  if (p2z_num_batches(from) < 0 || p2z_num_batches(to) < 0)
    return context_fail(ctx, P2Z_BAD_ARG, p2z_last_error(nullptr));
  if (from->nevts != to->nevts || from->nlayer != to->nlayer)
    return context_fail(ctx, P2Z_BAD_ARG, "from and to differ in nevts or nlayer");
  if ((mask_in == nullptr) != (mask_out == nullptr))
    return context_fail(ctx, P2Z_BAD_ARG, "pass both masks or neither");
  std::vector<int64_t> nf, nt;
  event_counts(from, nf);
  event_counts(to, nt);
  for (size_t e = 0; e < nf.size(); ++e) {
    if (nf[e] != nt[e]) {
      std::snprintf(msg, sizeof msg, "event %zu has %lld tracks in from and %lld in to", e, (long long)nf[e],
                    (long long)nt[e]);
      return context_fail(ctx, P2Z_BAD_ARG, msg);
    }
  }
  const int nev = (int)from->nevts;
  if (from->nevts > (1LL << 30)) return context_fail(ctx, P2Z_BAD_ARG, "too many events");
  const std::vector<int64_t> bf = event_begins(nf, from->bsize), bt = event_begins(nt, to->bsize);
  const int64_t nsf = bf.back(), nst = bt.back();
  if (nst == 0 || nev == 0) return P2Z_OK;
  if (!trk_in || !hits_in || !trk_out || !hits_out) return context_fail(ctx, P2Z_BAD_ARG, "NULL device buffer");
  // event tables: counts, source begins, destination begins
  void *tab = nullptr;
  TUNE_CUDA(ctx, scr.alloc(&tab, sizeof(int64_t) * (3 * (size_t)nev + 2)));
  int64_t *d_counts = (int64_t *)tab, *d_bf = d_counts + nev, *d_bt = d_bf + nev + 1;
  // the tables are read by the kernels below on st; host vectors outlive the
  // copies because the call synchronises st before returning
  TUNE_CUDA(ctx, cudaMemcpyAsync(d_counts, nf.data(), sizeof(int64_t) * nev, cudaMemcpyHostToDevice, st));
  TUNE_CUDA(ctx, cudaMemcpyAsync(d_bf, bf.data(), sizeof(int64_t) * (nev + 1), cudaMemcpyHostToDevice, st));
  TUNE_CUDA(ctx, cudaMemcpyAsync(d_bt, bt.data(), sizeof(int64_t) * (nev + 1), cudaMemcpyHostToDevice, st));
  const Side sf{from->bsize, from->layout == P2Z_LAYOUT_SOA ? 1 : 0, nsf, d_bf};
  const Side stt{to->bsize, to->layout == P2Z_LAYOUT_SOA ? 1 : 0, nst, d_bt};
  const unsigned gx = (unsigned)((nst + 255) / 256);
  k_relayout<<<dim3(gx, TRK_WORDS), 256, 0, st>>>((const uint32_t *)trk_in, (uint32_t *)trk_out, sf, stt, d_counts,
                                                    nev, ARR_TRK, from->nlayer);
  k_relayout<<<dim3(gx, HIT_WORDS * from->nlayer), 256, 0, st>>>((const uint32_t *)hits_in, (uint32_t *)hits_out, sf,
                                                                   stt, d_counts, nev, ARR_HIT, from->nlayer);
  if (mask_in)
    k_relayout<<<dim3(gx, 1), 256, 0, st>>>(mask_in, mask_out, sf, stt, d_counts, nev, ARR_MASK, from->nlayer);
  TUNE_CUDA(ctx, cudaGetLastError());
  TUNE_CUDA(ctx, cudaStreamSynchronize(st));
  return P2Z_OK;
}

}  // namespace

extern "C" {

p2z_status p2z_relayout_device(p2z_context *ctx, const p2z_config *from, const p2z_config *to, const void *d_trk_in,
                               const void *d_hits_in, const uint32_t *d_mask_in, void *d_trk_out, void *d_hits_out,
                               uint32_t *d_mask_out, void *stream) {
  if (!ctx) {
    set_context_free_error("context is NULL");
    return P2Z_BAD_ARG;
  }
  if (!from || !to) return context_fail(ctx, P2Z_BAD_ARG, "config is NULL");
  TUNE_CUDA(ctx, cudaSetDevice(context_device(ctx)));
  Scratch scr;
  return relayout(ctx, from, to, d_trk_in, d_hits_in, d_mask_in, d_trk_out, d_hits_out, d_mask_out,
                  stream ? (cudaStream_t)stream : context_stream(ctx), scr);
}

p2z_status p2z_autotune(p2z_context *ctx, const p2z_config *cfg, const void *d_trk_in, const void *d_hits,
                        const uint32_t *d_hit_mask, int reps, p2z_tune_entry *entries, int max_entries,
                        int *n_entries, p2z_tune_entry *best) {
  if (!ctx) {
    set_context_free_error("context is NULL");
    return P2Z_BAD_ARG;
  }
  if (!cfg) return context_fail(ctx, P2Z_BAD_ARG, "config is NULL");
  if (p2z_num_batches(cfg) < 0) return context_fail(ctx, P2Z_BAD_ARG, p2z_last_error(nullptr));
  if (max_entries < 0 || (max_entries > 0 && !entries)) return context_fail(ctx, P2Z_BAD_ARG, "bad entries array");
  if (reps <= 0) reps = 3;
  if (n_entries) *n_entries = 0;
  if (best) std::memset(best, 0, sizeof *best);
  TUNE_CUDA(ctx, cudaSetDevice(context_device(ctx)));
  cudaStream_t st = context_stream(ctx);
  std::vector<int64_t> counts;
  event_counts(cfg, counts);
  const bool masked = d_hit_mask != nullptr;
  const int nl = cfg->nlayer;
  static const int kB[] = {8, 16, 32, 64};
  static const int kBlock[] = {32, 64, 128, 256};
  std::vector<int> scheds = {P2Z_SCHED_FLAT, P2Z_SCHED_PERSISTENT};
  if (cfg->nevts <= 4096) scheds.push_back(P2Z_SCHED_PER_EVENT);
  // two threads per track: the precise 2-D update, every schedule but STAGED
  const bool pair_ok = cfg->update == P2Z_UPDATE_V2 && !(cfg->flags & P2Z_FLAG_REFERENCE_ROUNDING);

  // candidate configs per bsize: uniform when ntrks divides, else uneven with
  // the same per-event counts
  size_t max_trk = 0, max_hit = 0, max_slots = 0;
  for (int B : kB) {
    const int64_t ns = event_begins(counts, B).back();
    max_slots = std::max(max_slots, (size_t)ns);
    max_trk = std::max(max_trk, (size_t)ns * TRK_WORDS * 4);
    max_hit = std::max(max_hit, (size_t)ns * HIT_WORDS * nl * 4);
  }
  if (max_slots == 0) return P2Z_OK;
  if (!d_trk_in || !d_hits) return context_fail(ctx, P2Z_BAD_ARG, "NULL device buffer");
  Scratch scr;
  void *T = nullptr, *H = nullptr, *O = nullptr, *M = nullptr;
  TUNE_CUDA(ctx, scr.alloc(&T, max_trk));
  TUNE_CUDA(ctx, scr.alloc(&H, max_hit));
  TUNE_CUDA(ctx, scr.alloc(&O, max_trk));
  if (masked) TUNE_CUDA(ctx, scr.alloc(&M, max_slots * 4));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  TUNE_CUDA(ctx, cudaEventCreate(&e0));
  TUNE_CUDA(ctx, cudaEventCreate(&e1));
  struct EvGuard {
    cudaEvent_t a, b;
    ~EvGuard() {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
  } guard{e0, e1};

  int n = 0;
  p2z_tune_entry top;
  std::memset(&top, 0, sizeof top);
  top.ms = -1.0;
  for (int B : kB) {
    p2z_config c = *cfg;
    c.bsize = B;
    c.niter = 1;
    if (!cfg->event_ntrks && cfg->ntrks % B == 0) {
      c.event_ntrks = nullptr;
    } else {
      c.event_ntrks = counts.data();
    }
    for (int layout : {(int)P2Z_LAYOUT_AOSOA, (int)P2Z_LAYOUT_SOA}) {
      c.layout = layout;
      std::vector<int> sch = scheds;
      if (B == 32 && layout == P2Z_LAYOUT_AOSOA) sch.push_back(P2Z_SCHED_STAGED);
      p2z_status r = relayout(ctx, cfg, &c, d_trk_in, d_hits, d_hit_mask, T, H, (uint32_t *)M, st, scr);
      if (r != P2Z_OK) return r;
      // present-hit updates of one pass
      p2z_config cu = c;
      cu.schedule = P2Z_SCHED_FLAT;
      cu.block_threads = 128;
      cu.threads_per_track = 1;
      p2z_stats s0;
      r = p2z_run_device(ctx, &cu, T, H, (const uint32_t *)M, O, st, &s0);
      if (r != P2Z_OK) return r;
      p2z_tune_entry local;
      std::memset(&local, 0, sizeof local);
      local.ms = -1.0;
      // every (schedule, threads per track, window sorting, block size) of this bsize and layout;
      // window sorting applies to masked runs on the flat and persistent schedules
      struct Shape {
        int sched, tpt, sort, block;
      };
      std::vector<Shape> shapes;
      for (int sched : sch)
        for (int tpt = 1; tpt <= ((pair_ok && sched != P2Z_SCHED_STAGED) ? 2 : 1); ++tpt)
          for (int sort = 0;
               sort <= ((masked && (sched == P2Z_SCHED_FLAT || sched == P2Z_SCHED_PERSISTENT)) ? 1 : 0); ++sort)
            for (int block : kBlock) shapes.push_back({sched, tpt, sort, block});
      for (const Shape &sh : shapes) {
        c.schedule = sh.sched;
        c.block_threads = sh.block;
        c.threads_per_track = sh.tpt;
        c.flags = sh.sort ? (cfg->flags | P2Z_FLAG_SORT_WINDOWS) : (cfg->flags & ~P2Z_FLAG_SORT_WINDOWS);
        r = p2z_run_device(ctx, &c, T, H, (const uint32_t *)M, O, st, nullptr);  // warm-up (graph capture)
        if (r != P2Z_OK) return r;
        TUNE_CUDA(ctx, cudaEventRecord(e0, st));
        for (int i = 0; i < reps; ++i) {
          r = p2z_run_device(ctx, &c, T, H, (const uint32_t *)M, O, st, nullptr);
          if (r != P2Z_OK) return r;
        }
        TUNE_CUDA(ctx, cudaEventRecord(e1, st));
        TUNE_CUDA(ctx, cudaEventSynchronize(e1));
        float ms = 0.f;
        TUNE_CUDA(ctx, cudaEventElapsedTime(&ms, e0, e1));
        p2z_tune_entry t;
        std::memset(&t, 0, sizeof t);
        t.bsize = B;
        t.layout = layout;
        t.schedule = sh.sched;
        t.block_threads = sh.block;
        t.threads_per_track = sh.tpt;
        t.flags = sh.sort ? P2Z_FLAG_SORT_WINDOWS : 0u;
        t.ms = ms / reps;
        t.updates_per_s = t.ms > 0 ? (double)s0.updates / (t.ms * 1e-3) : 0.0;
        if (n < max_entries) entries[n] = t;
        ++n;
        if (local.ms < 0 || t.ms < local.ms) local = t;
      }
      c.schedule = P2Z_SCHED_AUTO;
      c.block_threads = 0;
      c.threads_per_track = 0;
      c.flags = cfg->flags;
      r = record_tuned(ctx, &c, masked, local.block_threads, local.schedule, local.threads_per_track,
                       (local.flags & P2Z_FLAG_SORT_WINDOWS) != 0);
      if (r != P2Z_OK) return r;
      if (top.ms < 0 || local.ms < top.ms) top = local;
    }
  }
  if (n_entries) *n_entries = n;
  if (best) *best = top;
  return P2Z_OK;
}

}  // extern "C"
