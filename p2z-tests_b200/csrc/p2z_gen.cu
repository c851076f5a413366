// p2z_gen.cu -- the physics workload generator and the layer-mask generator
// on the device: one thread per track slot, the same per-slot code as the host
// generator (p2z_gen.h).  The reference prepares its inputs on the host
// (prepareTracks / prepareHits, src/propagate-toz-test_OMP.cpp:243-293), which
// costs more than its timed region (4.4 s of setup against 0.77 s,
// logs/propagate_gcc_omp.log:27-28); generating the physics sample where it
// is consumed removes the host generation and the host->device copy.
#include <cuda_runtime.h>

#include <cstdio>
#include <vector>

#include "p2z.h"
#include "p2z_gen.h"

namespace p2z {
void set_context_free_error(const char *msg);
int context_device(const p2z_context *ctx);
cudaStream_t context_stream(const p2z_context *ctx);
p2z_status context_fail(p2z_context *ctx, p2z_status st, const char *msg);
void *context_scratch(p2z_context *ctx, size_t bytes);
}  // namespace p2z

using namespace p2z;

namespace {

// Slot s: the event it belongs to (last e with ev_first[e] <= s), real if
// s - ev_first[e] < ev_n[e], padding otherwise.
__global__ void __launch_bounds__(128) k_generate(p2z_physics_params p, double kf, int B, int nlayer, int64_t nslots,
                                                  int nevts, const int64_t *__restrict__ ev_first,
                                                  const int64_t *__restrict__ ev_n, float *trk, float *hits,
                                                  uint32_t *mask, uint32_t all) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslots) return;
  int lo = 0, hi = nevts - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (ev_first[mid] <= s) lo = mid;
    else hi = mid - 1;
  }
  const int64_t b = s / B;
  const p2z_gen::SlotView v{trk + b * (int64_t)p2z_gen::TRK_WORDS * B,
                            hits + b * nlayer * (int64_t)p2z_gen::HIT_WORDS * B, (int)(s % B), B};
  if (s - ev_first[lo] >= ev_n[lo]) {
    p2z_gen::zero_slot(nlayer, v);
    if (mask) mask[s] = 0u;
    return;
  }
  p2z_gen::generate_slot(p, kf, nlayer, (uint64_t)s, v);
  if (mask) mask[s] = all;
}

__global__ void k_mask_layers(uint32_t *mask, int64_t nslots, int min_hits, int max_hits, double drop_prob,
                              uint64_t seed) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslots || mask[s] == 0u) return;
  mask[s] = p2z_gen::mask_slot(seed, (uint64_t)s, min_hits, max_hits, drop_prob);
}

#define GEN_CUDA(ctx, call)                                                                      \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) {                                                                     \
      char m_[300];                                                                              \
      std::snprintf(m_, sizeof m_, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__,  \
                    __LINE__);                                                                   \
      return context_fail((ctx), P2Z_CUDA_ERROR, m_);                                            \
    }                                                                                            \
  } while (0)

}  // namespace

extern "C" {

p2z_status p2z_generate_physics_device(p2z_context *ctx, const p2z_physics_params *p, const p2z_config *cfg,
                                       void *d_trk_out, void *d_hits_out, uint32_t *d_hit_mask, void *stream) {
  if (!ctx) {
    set_context_free_error("context is NULL");
    return P2Z_BAD_ARG;
  }
  if (!p || !cfg) return context_fail(ctx, P2Z_BAD_ARG, "NULL argument");
  if (p2z_num_batches(cfg) < 0) return context_fail(ctx, P2Z_BAD_ARG, p2z_last_error(nullptr));
  if (cfg->layout != P2Z_LAYOUT_AOSOA) return context_fail(ctx, P2Z_UNSUPPORTED, "AOSOA layout only");
  if (p->pt_min <= 0 || p->pt_max < p->pt_min || p->eta_max < p->eta_min)
    return context_fail(ctx, P2Z_BAD_ARG, "physics parameters out of range");
  const int B = cfg->bsize, nlayer = cfg->nlayer;
  const int64_t nev = cfg->nevts;
  if (nev > (1LL << 30)) return context_fail(ctx, P2Z_BAD_ARG, "too many events");
  std::vector<int64_t> tab(2 * (size_t)nev + 1, 0);  // ev_first[nev + 1], ev_n[nev]
  int64_t nb = 0;
  for (int64_t e = 0; e < nev; ++e) {
    const int64_t n = cfg->event_ntrks ? cfg->event_ntrks[e] : cfg->ntrks;
    tab[e] = nb * B;
    tab[nev + 1 + e] = n;
    nb += (n + B - 1) / B;
  }
  tab[nev] = nb * B;
  const int64_t nslots = nb * B;
  if (nslots == 0) return P2Z_OK;
  if (!d_trk_out || !d_hits_out) return context_fail(ctx, P2Z_BAD_ARG, "NULL device buffer");
  GEN_CUDA(ctx, cudaSetDevice(context_device(ctx)));
  cudaStream_t st = stream ? (cudaStream_t)stream : context_stream(ctx);
  int64_t *d_tab = (int64_t *)context_scratch(ctx, sizeof(int64_t) * tab.size());
  if (!d_tab) return context_fail(ctx, P2Z_OOM, "generator scratch allocation failed");
  GEN_CUDA(ctx, cudaMemcpyAsync(d_tab, tab.data(), sizeof(int64_t) * tab.size(), cudaMemcpyHostToDevice, st));
  const double kf = p->kfact != 0.f ? p->kfact : (double)(float)(100. / (-0.299792458 * 3.8112));
  const uint32_t all = nlayer >= 32 ? 0xffffffffu : ((1u << nlayer) - 1u);
  k_generate<<<(unsigned)((nslots + 127) / 128), 128, 0, st>>>(*p, kf, B, nlayer, nslots, (int)nev, d_tab,
                                                               d_tab + nev + 1, (float *)d_trk_out,
                                                               (float *)d_hits_out, d_hit_mask, all);
  GEN_CUDA(ctx, cudaGetLastError());
  GEN_CUDA(ctx, cudaStreamSynchronize(st));  // the event table's host copy dies with this call
  return P2Z_OK;
}

p2z_status p2z_mask_layers_device(p2z_context *ctx, uint32_t *d_hit_mask, int64_t nslots, int nlayer, int min_hits,
                                  int max_hits, double drop_prob, uint64_t seed, void *stream) {
  if (!ctx) {
    set_context_free_error("context is NULL");
    return P2Z_BAD_ARG;
  }
  if ((!d_hit_mask && nslots > 0) || nslots < 0) return context_fail(ctx, P2Z_BAD_ARG, "bad mask array");
  if (nlayer < 1 || nlayer > 32 || min_hits < 1 || max_hits < min_hits || max_hits > nlayer || drop_prob < 0 ||
      drop_prob >= 1)
    return context_fail(ctx, P2Z_BAD_ARG, "mask parameters out of range");
  if (nslots == 0) return P2Z_OK;
  GEN_CUDA(ctx, cudaSetDevice(context_device(ctx)));
  cudaStream_t st = stream ? (cudaStream_t)stream : context_stream(ctx);
  k_mask_layers<<<(unsigned)((nslots + 255) / 256), 256, 0, st>>>(d_hit_mask, nslots, min_hits, max_hits, drop_prob,
                                                                  seed);
  GEN_CUDA(ctx, cudaGetLastError());
  return P2Z_OK;
}

}  // extern "C"
