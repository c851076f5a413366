// p2z_serve.cu -- continuous-batching server (include/p2z.h, "serving").
//
// Device memory: one slot ring sized by the budget, made of parallel arrays
// indexed by a batch number b in [0, capacity): track batches (in and out),
// nlayer hit batches per track batch, one mask word per slot.  An event of n
// tracks occupies ceil(n/bsize) consecutive batches, so a group of events
// admitted one after another is one contiguous slot range for the kernel.
// Ring space is handed out at the head and given back at the tail, in
// completion order (groups complete in launch order).
//
// One scheduler thread owns every CUDA call: it admits events (host->device
// copies on the copy stream), launches groups (the persistent kernel on the
// compute stream after the group's copies), reads each event back on the
// compute stream followed by a per-event completion event, and polls those
// events to retire requests.  Submitting threads only touch the request table
// under the mutex.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "p2z.h"
#include "p2z_kernels.cuh"

using namespace p2z;

namespace {

cudaError_t dispatch_kernel(const LaunchSpec &s, cudaStream_t st) {
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

int kernel_occupancy(const LaunchSpec &s) {
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

// Masks of an event submitted without one: every layer for real lanes, 0 for
// the padding lanes of its last batch.
__global__ void k_event_mask(uint32_t *mask, int64_t slot0, int64_t nslots, int64_t nreal, uint32_t all) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nslots) return;
  mask[slot0 + i] = (i < nreal) ? all : 0u;
}

enum class St { Pending, Admitted, Launched, Done };

struct Request {
  int64_t id = 0;
  const void *trk_in = nullptr;
  const void *hits = nullptr;
  const uint32_t *mask = nullptr;
  void *trk_out = nullptr;
  int64_t ntrks = 0, nb = 0;
  int64_t b0 = -1;  // first ring batch
  St st = St::Pending;
  cudaEvent_t done_ev = nullptr;
  int group = -1;
  p2z_request_info info{};
};

double now_s(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

struct p2z_server {
  p2z_server_config cfg{};
  int device = 0;
  int num_sms = 0;
  int upd = UPDK_V2;
  int sc = SC_FAST;
  int64_t cap = 0;  // ring capacity in batches
  size_t trk_b = 0, hit_b = 0;
  float *d_trk = nullptr, *d_out = nullptr, *d_hit = nullptr;
  uint32_t *d_mask = nullptr;
  unsigned long long *d_counters = nullptr;  // one persistent work counter per group slot
  unsigned int *d_status = nullptr;
  cudaStream_t copy = nullptr, compute = nullptr;
  cudaEvent_t copied = nullptr;  // a group's copies issued (re-recorded for every group)
  int occupancy = 0;             // resident CTAs per SM of the server's kernel (fixed per server)
  int max_inflight = 2;

  // ring
  int64_t head = 0, tail = 0, used = 0;  // used counts batches including wrap waste
  std::deque<std::pair<int64_t, int64_t>> live;  // (b0, nb incl. waste) in allocation order

  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::unordered_map<int64_t, Request> reqs;
  std::deque<int64_t> pending, admitted;  // ids in order
  std::deque<std::vector<int64_t>> inflight;  // launched groups in order
  std::vector<cudaEvent_t> free_events;
  int64_t next_id = 1;
  int group_seq = 0;
  bool stop = false;
  std::thread worker;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

  // ---- ring allocation (scheduler thread, mutex held) ------------------------
  // Live batches are [tail, head) when head > tail, [tail, cap) + [0, head)
  // when head < tail, everything when head == tail and used > 0.  `live` lists
  // the allocations (and wasted ring ends) in allocation order.
  bool ring_alloc(int64_t nb, int64_t *b0) {
    if (nb > cap) return false;
    if (used == 0) head = tail = 0;
    if (cap - used < nb) return false;
    if (used == 0 || head > tail) {
      if (head + nb <= cap) {
        *b0 = head;
      } else if (nb <= tail) {
        live.emplace_back(head, cap - head);  // the end of the ring stays unused
        used += cap - head;
        *b0 = 0;
      } else {
        return false;
      }
    } else {
      if (head == tail || head + nb > tail) return false;  // full, or the gap is too small
      *b0 = head;
    }
    live.emplace_back(*b0, nb);
    used += nb;
    head = (*b0 + nb) % cap;
    return true;
  }
};

namespace {

// Admit pending requests into the ring (mutex held).
void admit(p2z_server *s) {
  const int B = s->cfg.bsize, nl = s->cfg.nlayer;
  const bool six = (s->upd == UPDK_V2 || s->upd == UPDK_V2_COMP || s->upd == UPDK_F64 || s->upd == UPDK_V2_REF) &&
                   !(s->cfg.flags & P2Z_FLAG_FULL_HITS);
  const uint32_t all = nl >= 32 ? 0xffffffffu : ((1u << nl) - 1u);
  while (!s->pending.empty()) {
    Request &r = s->reqs[s->pending.front()];
    int64_t b0;
    if (!s->ring_alloc(r.nb, &b0)) break;
    r.b0 = b0;
    const size_t trk_bytes = s->trk_b * (size_t)r.nb;
    cudaMemcpyAsync((char *)s->d_trk + b0 * s->trk_b, r.trk_in, trk_bytes, cudaMemcpyHostToDevice, s->copy);
    const size_t hrows = (size_t)r.nb * nl;
    char *hdst = (char *)s->d_hit + (size_t)b0 * nl * s->hit_b;
    if (six)
      cudaMemcpy2DAsync(hdst, s->hit_b, r.hits, s->hit_b, 6 * (size_t)B * 4, hrows, cudaMemcpyHostToDevice, s->copy);
    else
      cudaMemcpyAsync(hdst, r.hits, s->hit_b * hrows, cudaMemcpyHostToDevice, s->copy);
    const int64_t slot0 = b0 * B, nslots = r.nb * B;
    if (r.mask) {
      cudaMemcpyAsync(s->d_mask + slot0, r.mask, nslots * 4, cudaMemcpyHostToDevice, s->copy);
    } else {
      k_event_mask<<<(unsigned)((nslots + 255) / 256), 256, 0, s->copy>>>(s->d_mask, slot0, nslots, r.ntrks, all);
    }
    r.st = St::Admitted;
    r.info.admit_s = now_s(s->t0);
    s->admitted.push_back(r.id);
    s->pending.pop_front();
  }
}

// Launch every admitted request as one group (mutex held).
void launch_group(p2z_server *s) {
  if (s->admitted.empty() || (int)s->inflight.size() >= s->max_inflight) return;
  const int B = s->cfg.bsize;
  const int slot_idx = s->group_seq % 8;
  s->group_seq++;
  std::vector<int64_t> ids(s->admitted.begin(), s->admitted.end());
  s->admitted.clear();
  // the group's copies were issued on the copy stream before this point
  cudaEventRecord(s->copied, s->copy);
  cudaStreamWaitEvent(s->compute, s->copied, 0);
  // contiguous runs of ring batches (a run breaks where the ring wraps)
  LaunchSpec spec;
  std::memset(&spec, 0, sizeof spec);
  spec.tpt = 1;
  spec.args.trk = s->d_trk;
  spec.args.hits = s->d_hit;
  spec.args.out = s->d_out;
  spec.args.mask = s->d_mask;
  spec.args.nlayer = s->cfg.nlayer;
  spec.args.kfact = s->cfg.kfact != 0.f ? s->cfg.kfact : (float)(100. / (-0.299792458 * 3.8112));
  spec.args.status = s->d_status;
  spec.args.queue = s->d_counters + slot_idx;
  spec.bsize = B;
  spec.upd = s->upd;
  spec.sc = s->sc;
  spec.masked = true;
  spec.kind = KIND_PERSISTENT;
  spec.block = s->cfg.block_threads ? s->cfg.block_threads : 128;
  if (s->occupancy == 0) s->occupancy = std::max(1, kernel_occupancy(spec));  // same kernel and block every group
  const int occ = s->occupancy;
  const double t = now_s(s->t0);
  size_t i = 0;
  while (i < ids.size()) {
    Request &first = s->reqs[ids[i]];
    int64_t b_begin = first.b0, b_end = first.b0 + first.nb;
    size_t j = i + 1;
    while (j < ids.size() && s->reqs[ids[j]].b0 == b_end) {
      b_end += s->reqs[ids[j]].nb;
      ++j;
    }
    spec.args.slot_begin = b_begin * B;
    spec.args.slot_end = b_end * B;
    // a run of at most 4 warps per SM asks L2 for its hit blocks first (as p2z_run_device)
    spec.args.l2_prefetch = (spec.args.slot_end - spec.args.slot_begin) <= (int64_t)s->num_sms * 4 * 32 ? 1 : 0;
    const int64_t items = (spec.args.slot_end - spec.args.slot_begin + 31) / 32;
    spec.grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)occ * s->num_sms, (items * 32 + spec.block - 1) /
                                                                                              spec.block));
    cudaMemsetAsync(spec.args.queue, 0, sizeof(unsigned long long), s->compute);
    dispatch_kernel(spec, s->compute);
    i = j;
  }
  // read each event back, then its completion event
  for (int64_t id : ids) {
    Request &r = s->reqs[id];
    cudaMemcpyAsync(r.trk_out, (const char *)s->d_out + r.b0 * s->trk_b, s->trk_b * (size_t)r.nb,
                    cudaMemcpyDeviceToHost, s->compute);
    if (s->free_events.empty()) {
      cudaEventCreateWithFlags(&r.done_ev, cudaEventDisableTiming);
    } else {
      r.done_ev = s->free_events.back();
      s->free_events.pop_back();
    }
    cudaEventRecord(r.done_ev, s->compute);
    r.st = St::Launched;
    r.info.launch_s = t;
    r.info.group_events = (int32_t)ids.size();
  }
  s->inflight.push_back(std::move(ids));
}

// Retire completed groups in order (mutex held).  Returns true if any retired.
bool retire(p2z_server *s) {
  bool any = false;
  while (!s->inflight.empty()) {
    std::vector<int64_t> &g = s->inflight.front();
    bool done = true;
    for (int64_t id : g) {
      if (cudaEventQuery(s->reqs[id].done_ev) != cudaSuccess) {
        done = false;
        break;
      }
    }
    if (!done) break;
    cudaGetLastError();
    const double t = now_s(s->t0);
    for (int64_t id : g) {
      Request &r = s->reqs[id];
      r.st = St::Done;
      r.info.done_s = t;
      r.info.status = P2Z_OK;
      s->free_events.push_back(r.done_ev);
      r.done_ev = nullptr;
      // give the ring space back: allocations were made in this same order
      while (!s->live.empty()) {
        auto front = s->live.front();
        s->live.pop_front();
        s->used -= front.second;
        s->tail = (front.first + front.second) % s->cap;
        if (front.first == r.b0 && front.second == r.nb) break;
      }
      if (s->used == 0) s->head = s->tail = 0;
    }
    s->inflight.pop_front();
    any = true;
  }
  return any;
}

void worker_loop(p2z_server *s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    const bool any = retire(s);
    admit(s);
    launch_group(s);
    if (any) s->cv_done.notify_all();
    if (s->stop && s->pending.empty() && s->admitted.empty() && s->inflight.empty()) break;
    if (s->inflight.empty() && s->pending.empty() && s->admitted.empty()) {
      s->cv_work.wait_for(lk, std::chrono::milliseconds(5));
    } else {
      // poll the GPU without holding the lock for long: yield for a few
      // microseconds (a sleep of that length lasts the OS timer slack, tens of
      // microseconds, which every request's latency would carry)
      lk.unlock();
      const auto until = std::chrono::steady_clock::now() + std::chrono::microseconds(5);
      while (std::chrono::steady_clock::now() < until) std::this_thread::yield();
      lk.lock();
    }
  }
  s->cv_done.notify_all();
}

}  // namespace

extern "C" {

p2z_status p2z_server_create(int device, const p2z_server_config *cfg, p2z_server **out) {
  if (!cfg || !out) return P2Z_BAD_ARG;
  *out = nullptr;
  if (cfg->abi_version != P2Z_ABI_VERSION) return P2Z_BAD_ARG;
  if (!(cfg->bsize == 8 || cfg->bsize == 16 || cfg->bsize == 32 || cfg->bsize == 64)) return P2Z_UNSUPPORTED;
  if (cfg->nlayer < 1 || cfg->nlayer > 32 || cfg->update < 0 || cfg->update > P2Z_UPDATE_F64) return P2Z_BAD_ARG;
  if (cfg->device_budget_bytes <= 0 || !std::isfinite(cfg->kfact)) return P2Z_BAD_ARG;
  if (cfg->block_threads != 0 && (cfg->block_threads < 32 || cfg->block_threads > 256 || cfg->block_threads % 32))
    return P2Z_BAD_ARG;
  if ((cfg->flags & P2Z_FLAG_REFERENCE_ROUNDING) && cfg->update != P2Z_UPDATE_V2) return P2Z_UNSUPPORTED;
  // the flags a group launch honours; the others (STRICT, CHECK_INPUTS, the schedule flags) have no
  // per-request status or launch form here
  if (cfg->flags & ~(uint32_t)(P2Z_FLAG_ACCURATE_TRIG | P2Z_FLAG_REFERENCE_ROUNDING | P2Z_FLAG_FULL_HITS))
    return P2Z_UNSUPPORTED;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return P2Z_NO_DEVICE;
  }
  if (device < 0) cudaGetDevice(&device);
  if (device >= ndev) return P2Z_BAD_ARG;
  p2z_server *s = new p2z_server();
  s->cfg = *cfg;
  s->device = device;
  s->upd = (cfg->flags & P2Z_FLAG_REFERENCE_ROUNDING) ? UPDK_V2_REF : cfg->update;
  s->sc = (cfg->flags & P2Z_FLAG_ACCURATE_TRIG) ? SC_ACCURATE : SC_FAST;
  // each group in flight uses its own persistent work counter (8 of them)
  s->max_inflight = cfg->max_inflight > 0 ? std::min(cfg->max_inflight, 8) : 2;
  const int B = cfg->bsize, nl = cfg->nlayer;
  s->trk_b = (size_t)TRK_WORDS * B * 4;
  s->hit_b = (size_t)HIT_WORDS * B * 4;
  const size_t per_batch = 2 * s->trk_b + (size_t)nl * s->hit_b + (size_t)B * 4;
  s->cap = (int64_t)(cfg->device_budget_bytes / (int64_t)per_batch);
  cudaError_t e;
  auto bail = [&](p2z_status st) {
    cudaGetLastError();
    p2z_server_destroy(s);
    return st;
  };
  if (s->cap < 1) return bail(P2Z_BAD_ARG);
  if ((e = cudaSetDevice(device)) != cudaSuccess) return bail(P2Z_CUDA_ERROR);
  cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, device);
  if ((e = cudaMalloc(&s->d_trk, s->trk_b * s->cap)) != cudaSuccess) return bail(P2Z_OOM);
  if ((e = cudaMalloc(&s->d_out, s->trk_b * s->cap)) != cudaSuccess) return bail(P2Z_OOM);
  if ((e = cudaMalloc(&s->d_hit, s->hit_b * nl * s->cap)) != cudaSuccess) return bail(P2Z_OOM);
  if ((e = cudaMalloc(&s->d_mask, (size_t)B * 4 * s->cap)) != cudaSuccess) return bail(P2Z_OOM);
  if ((e = cudaMalloc(&s->d_counters, 8 * sizeof(unsigned long long))) != cudaSuccess) return bail(P2Z_OOM);
  if ((e = cudaMalloc(&s->d_status, sizeof(unsigned int))) != cudaSuccess) return bail(P2Z_OOM);
  if ((e = cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking)) != cudaSuccess) return bail(P2Z_CUDA_ERROR);
  if ((e = cudaStreamCreateWithFlags(&s->compute, cudaStreamNonBlocking)) != cudaSuccess) return bail(P2Z_CUDA_ERROR);
  if ((e = cudaEventCreateWithFlags(&s->copied, cudaEventDisableTiming)) != cudaSuccess) return bail(P2Z_CUDA_ERROR);
  cudaMemset(s->d_status, 0, sizeof(unsigned int));
  s->worker = std::thread(worker_loop, s);
  *out = s;
  return P2Z_OK;
}

p2z_status p2z_server_destroy(p2z_server *s) {
  if (!s) return P2Z_OK;
  if (s->worker.joinable()) {
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->stop = true;
    }
    s->cv_work.notify_all();
    s->worker.join();
  }
  cudaSetDevice(s->device);
  if (s->compute) cudaStreamSynchronize(s->compute);
  if (s->copy) cudaStreamSynchronize(s->copy);
  for (auto &kv : s->reqs)
    if (kv.second.done_ev) cudaEventDestroy(kv.second.done_ev);
  for (cudaEvent_t ev : s->free_events) cudaEventDestroy(ev);
  if (s->copied) cudaEventDestroy(s->copied);
  for (void *p : {(void *)s->d_trk, (void *)s->d_out, (void *)s->d_hit, (void *)s->d_mask, (void *)s->d_counters,
                  (void *)s->d_status})
    if (p) cudaFree(p);
  if (s->copy) cudaStreamDestroy(s->copy);
  if (s->compute) cudaStreamDestroy(s->compute);
  delete s;
  return P2Z_OK;
}

double p2z_server_now(const p2z_server *s) { return s ? now_s(s->t0) : 0.0; }

p2z_status p2z_server_submit(p2z_server *s, const void *trk_in, const void *hits, const uint32_t *hit_mask,
                             int64_t ntrks, void *trk_out, int64_t *id) {
  if (!s || !id || ntrks < 0) return P2Z_BAD_ARG;
  if (ntrks > 0 && (!trk_in || !hits || !trk_out)) return P2Z_BAD_ARG;
  const int64_t nb = (ntrks + s->cfg.bsize - 1) / s->cfg.bsize;
  if (nb > s->cap) return P2Z_OOM;
  Request r;
  r.trk_in = trk_in;
  r.hits = hits;
  r.mask = hit_mask;
  r.trk_out = trk_out;
  r.ntrks = ntrks;
  r.nb = nb;
  r.info.ntrks = ntrks;
  const uint32_t all = s->cfg.nlayer >= 32 ? 0xffffffffu : ((1u << s->cfg.nlayer) - 1u);
  if (hit_mask) {
    int64_t u = 0;
    for (int64_t i = 0; i < ntrks; ++i) u += __builtin_popcount(hit_mask[i] & all);
    r.info.updates = u;
  } else {
    r.info.updates = ntrks * s->cfg.nlayer;
  }
  {
    std::lock_guard<std::mutex> lk(s->mu);
    r.id = s->next_id++;
    r.info.submit_s = now_s(s->t0);
    *id = r.id;
    if (nb == 0) {
      // an event without tracks has nothing to copy or compute: done at once
      r.st = St::Done;
      r.info.admit_s = r.info.launch_s = r.info.done_s = r.info.submit_s;
      r.info.status = P2Z_OK;
      s->reqs.emplace(r.id, r);
      return P2Z_OK;
    }
    s->reqs.emplace(r.id, r);
    s->pending.push_back(r.id);
  }
  s->cv_work.notify_all();
  return P2Z_OK;
}

p2z_status p2z_server_poll(p2z_server *s, int64_t id, p2z_request_info *info) {
  if (!s) return P2Z_BAD_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return P2Z_BAD_ARG;
  if (it->second.st != St::Done) return P2Z_NOT_READY;
  if (info) *info = it->second.info;
  s->reqs.erase(it);  // a completed request is released once reported
  return P2Z_OK;
}

p2z_status p2z_server_wait(p2z_server *s, int64_t id, double timeout_s, p2z_request_info *info) {
  if (!s) return P2Z_BAD_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout_s);
  for (;;) {
    // look the request up after every wake-up: submits from other threads may
    // have rehashed the table meanwhile
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return P2Z_BAD_ARG;
    if (it->second.st == St::Done) {
      if (info) *info = it->second.info;
      s->reqs.erase(it);  // a completed request is released once reported
      return P2Z_OK;
    }
    if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout) {
      auto again = s->reqs.find(id);
      if (again == s->reqs.end()) return P2Z_BAD_ARG;
      if (again->second.st != St::Done) return P2Z_TIMEOUT;
    }
  }
}

p2z_status p2z_server_replay(p2z_server *s, int64_t nreq, const void *const *trk_in, const void *const *hits,
                             const uint32_t *const *hit_mask, const int64_t *ntrks, void *const *trk_out,
                             const double *arrival_s, p2z_request_info *infos) {
  if (!s || nreq < 0 || (nreq > 0 && (!trk_in || !hits || !ntrks || !trk_out || !arrival_s || !infos)))
    return P2Z_BAD_ARG;
  std::vector<int64_t> ids(nreq);
  const double start = p2z_server_now(s);
  for (int64_t i = 0; i < nreq; ++i) {
    const double due = start + arrival_s[i];
    double t;
    while ((t = p2z_server_now(s)) < due) {
      if (due - t > 200e-6) std::this_thread::sleep_for(std::chrono::duration<double>((due - t) - 100e-6));
    }
    p2z_status st =
        p2z_server_submit(s, trk_in[i], hits[i], hit_mask ? hit_mask[i] : nullptr, ntrks[i], trk_out[i], &ids[i]);
    if (st != P2Z_OK) return st;
  }
  for (int64_t i = 0; i < nreq; ++i) {
    p2z_status st = p2z_server_wait(s, ids[i], 600.0, &infos[i]);
    if (st != P2Z_OK) return st;
  }
  return P2Z_OK;
}

}  // extern "C"
