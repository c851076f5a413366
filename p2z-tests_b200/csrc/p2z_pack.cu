// p2z_pack.cu -- packing an uneven sample in order of hit count on the device.
//
// A warp's 32 tracks take as many steps as the one with the most hits, so
// tracks with missing layers run fastest when each batch holds tracks of
// similar hit counts.  p2z_pack_by_hits_device writes a copy of the arrays in
// which every event's tracks are in order of decreasing hit count (equal
// counts keep their order; each event keeps its slots, padding last), plus the
// permutation; p2z_unpack_tracks_device puts a packed output back in the
// caller's order.  No counterpart in the reference, whose events hold every
// layer of every track (src/propagate-toz-test_OMP.cpp:731-748).
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>

#include <cstdio>
#include <vector>

#include "p2z.h"
#include "p2z_kernels.cuh"

namespace p2z {
void set_context_free_error(const char *msg);
int context_device(const p2z_context *ctx);
cudaStream_t context_stream(const p2z_context *ctx);
p2z_status context_fail(p2z_context *ctx, p2z_status st, const char *msg);
void *context_scratch(p2z_context *ctx, size_t bytes);
}  // namespace p2z

using namespace p2z;

namespace {

#define PACK_CUDA(ctx, call)                                                                    \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) {                                                                    \
      char m_[300];                                                                             \
      std::snprintf(m_, sizeof m_, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                    __LINE__);                                                                  \
      return context_fail((ctx), e_ == cudaErrorMemoryAllocation ? P2Z_OOM : P2Z_CUDA_ERROR, m_); \
    }                                                                                           \
  } while (0)

size_t up256(size_t n) { return (n + 255) / 256 * 256; }

// Sort key of slot s: (event << 6) | rank class, where the class is
// 32 - (hit count) for a real track (0: every one of 32 layers present) and
// 33 for a padding slot, so that each event keeps its slots and its padding
// stays last.  counts: real tracks per event; beg: first slot of each event.
__global__ void k_pack_keys(const uint32_t *__restrict__ mask, const int64_t *__restrict__ beg,
                            const int64_t *__restrict__ counts, int nevts, int64_t nslots, uint32_t all,
                            uint64_t *__restrict__ keys, int64_t *__restrict__ idx) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslots) return;
  int lo = 0, hi = nevts - 1;  // event of s: the last e with beg[e] <= s
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (beg[mid] <= s) lo = mid;
    else hi = mid - 1;
  }
  const bool real = s - beg[lo] < counts[lo];
  const uint32_t m = mask ? (__ldg(mask + s) & all) : all;
  const uint64_t cls = real ? (uint64_t)(32 - __popc(m)) : 33u;
  keys[s] = ((uint64_t)lo << 6) | cls;
  idx[s] = s;
}

// One slot's words in an AOSOA array whose batches are `bw` words long (28 B
// for tracks; nlayer * 9 * B for hits, whose layers of a batch are
// contiguous): word r of slot s is at (s / B) * bw + s % B + r * B.
__device__ __forceinline__ int64_t slot_base(int64_t s, int B, int64_t bw) { return (s / B) * bw + s % B; }

// Thread = destination slot s, copying all `rows` words of a slot: dst[s] =
// src[perm[s]] (packing with the permutation, unpacking with its inverse).
// Consecutive threads write consecutive slots.
__global__ void k_gather(const uint32_t *__restrict__ src, uint32_t *__restrict__ dst,
                         const int64_t *__restrict__ perm, int64_t nslots, int B, int rows, int64_t bw) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslots) return;
  const int64_t from = slot_base(perm[s], B, bw), to = slot_base(s, B, bw);
#pragma unroll 4
  for (int r = 0; r < rows; ++r) dst[to + (int64_t)r * B] = src[from + (int64_t)r * B];
}

// inv[perm[s]] = s
__global__ void k_invert(const int64_t *__restrict__ perm, int64_t *__restrict__ inv, int64_t nslots) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s < nslots) inv[perm[s]] = s;
}

__global__ void k_gather_mask(const uint32_t *__restrict__ src, uint32_t *__restrict__ dst,
                              const int64_t *__restrict__ perm, int64_t nslots) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s < nslots) dst[s] = src[perm[s]];
}

// Event tables of a config: per-event real tracks and first slots (nevts + 1).
void event_tables(const p2z_config *c, std::vector<int64_t> &counts, std::vector<int64_t> &beg) {
  const int64_t ne = c->nevts;
  counts.assign((size_t)ne, 0);
  beg.assign((size_t)ne + 1, 0);
  for (int64_t e = 0; e < ne; ++e) {
    counts[e] = c->event_ntrks ? c->event_ntrks[e] : c->ntrks;
    beg[e + 1] = beg[e] + (counts[e] + c->bsize - 1) / c->bsize * c->bsize;
  }
}

p2z_status check_config(p2z_context *ctx, const p2z_config *cfg, int64_t *nslots) {
  if (!cfg) return context_fail(ctx, P2Z_BAD_ARG, "config is NULL");
  const int64_t nb = p2z_num_batches(cfg);
  if (nb < 0) return context_fail(ctx, P2Z_BAD_ARG, p2z_last_error(nullptr));
  if (cfg->layout != P2Z_LAYOUT_AOSOA) return context_fail(ctx, P2Z_UNSUPPORTED, "packing needs the AOSOA layout");
  if (cfg->nevts >= (1LL << 30)) return context_fail(ctx, P2Z_BAD_ARG, "too many events");
  *nslots = nb * cfg->bsize;
  return P2Z_OK;
}

}  // namespace

extern "C" {

p2z_status p2z_pack_by_hits_device(p2z_context *ctx, const p2z_config *cfg, const void *d_trk_in,
                                   const void *d_hits_in, const uint32_t *d_mask_in, void *d_trk_out,
                                   void *d_hits_out, uint32_t *d_mask_out, int64_t *d_perm, void *stream) {
  if (!ctx) {
    set_context_free_error("context is NULL");
    return P2Z_BAD_ARG;
  }
  int64_t ns = 0;
  p2z_status r = check_config(ctx, cfg, &ns);
  if (r != P2Z_OK) return r;
  if ((d_mask_in == nullptr) != (d_mask_out == nullptr))
    return context_fail(ctx, P2Z_BAD_ARG, "pass both masks or neither");
  if (ns == 0) return P2Z_OK;
  if (!d_trk_in || !d_hits_in || !d_trk_out || !d_hits_out || !d_perm)
    return context_fail(ctx, P2Z_BAD_ARG, "NULL device buffer");
  if (d_trk_in == d_trk_out || d_hits_in == d_hits_out || (d_mask_in && d_mask_in == d_mask_out))
    return context_fail(ctx, P2Z_BAD_ARG, "the packed copy must not alias the input");
  PACK_CUDA(ctx, cudaSetDevice(context_device(ctx)));
  cudaStream_t st = stream ? (cudaStream_t)stream : context_stream(ctx);
  std::vector<int64_t> counts, beg;
  event_tables(cfg, counts, beg);
  const int ne = (int)cfg->nevts;
  // the sort's bits: 6 for the class, then the event index
  int end_bit = 6;
  while (end_bit < 64 && ((uint64_t)ne - 1) >> (end_bit - 6)) ++end_bit;
  size_t tmp_bytes = 0;
  PACK_CUDA(ctx, cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, (const uint64_t *)nullptr, (uint64_t *)nullptr,
                                                 (const int64_t *)nullptr, (int64_t *)nullptr, ns, 0, end_bit, st));
  // scratch, from the context's reusable device buffer (parts 256-byte aligned): event tables,
  // keys, sorted keys, slot indices, the sort's temporary storage
  const size_t b_tab = up256(sizeof(int64_t) * (2 * (size_t)ne + 1)), b_keys = up256(sizeof(uint64_t) * (size_t)ns);
  char *scr = static_cast<char *>(context_scratch(ctx, b_tab + 3 * b_keys + up256(tmp_bytes)));
  if (!scr) return context_fail(ctx, P2Z_OOM, "no device memory for the packing scratch");
  void *tab = scr, *keys = scr + b_tab, *keys_sorted = scr + b_tab + b_keys, *idx = scr + b_tab + 2 * b_keys;
  void *tmp = scr + b_tab + 3 * b_keys;
  int64_t *d_counts = (int64_t *)tab, *d_beg = d_counts + ne;
  PACK_CUDA(ctx, cudaMemcpyAsync(d_counts, counts.data(), sizeof(int64_t) * ne, cudaMemcpyHostToDevice, st));
  PACK_CUDA(ctx, cudaMemcpyAsync(d_beg, beg.data(), sizeof(int64_t) * (ne + 1), cudaMemcpyHostToDevice, st));
  const uint32_t all = cfg->nlayer >= 32 ? 0xffffffffu : ((1u << cfg->nlayer) - 1u);
  const unsigned gx = (unsigned)((ns + 255) / 256);
  k_pack_keys<<<gx, 256, 0, st>>>(d_mask_in, d_beg, d_counts, ne, ns, all, (uint64_t *)keys, (int64_t *)idx);
  PACK_CUDA(ctx, cudaGetLastError());
  // stable radix sort of (event, class) over the bits the keys use
  PACK_CUDA(ctx, cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, (const uint64_t *)keys, (uint64_t *)keys_sorted,
                                                 (const int64_t *)idx, d_perm, ns, 0, end_bit, st));
  const int B = cfg->bsize, nl = cfg->nlayer;
  k_gather<<<gx, 256, 0, st>>>((const uint32_t *)d_trk_in, (uint32_t *)d_trk_out, d_perm, ns, B, TRK_WORDS,
                                      (int64_t)TRK_WORDS * B);
  k_gather<<<gx, 256, 0, st>>>((const uint32_t *)d_hits_in, (uint32_t *)d_hits_out, d_perm, ns, B,
                                      HIT_WORDS * nl, (int64_t)HIT_WORDS * nl * B);
  if (d_mask_in) k_gather_mask<<<gx, 256, 0, st>>>(d_mask_in, d_mask_out, d_perm, ns);
  k_invert<<<gx, 256, 0, st>>>(d_perm, d_perm + ns, ns);
  PACK_CUDA(ctx, cudaGetLastError());
  PACK_CUDA(ctx, cudaStreamSynchronize(st));
  return P2Z_OK;
}

p2z_status p2z_unpack_tracks_device(p2z_context *ctx, const p2z_config *cfg, const int64_t *d_perm,
                                    const void *d_trk_packed, void *d_trk_out, void *stream) {
  if (!ctx) {
    set_context_free_error("context is NULL");
    return P2Z_BAD_ARG;
  }
  int64_t ns = 0;
  p2z_status r = check_config(ctx, cfg, &ns);
  if (r != P2Z_OK) return r;
  if (ns == 0) return P2Z_OK;
  if (!d_perm || !d_trk_packed || !d_trk_out) return context_fail(ctx, P2Z_BAD_ARG, "NULL device buffer");
  if (d_trk_packed == d_trk_out) return context_fail(ctx, P2Z_BAD_ARG, "d_trk_out must not alias d_trk_packed");
  PACK_CUDA(ctx, cudaSetDevice(context_device(ctx)));
  cudaStream_t st = stream ? (cudaStream_t)stream : context_stream(ctx);
  const unsigned gx = (unsigned)((ns + 255) / 256);
  // a gather through the inverse permutation (d_perm's second half): the writes are coalesced
  k_gather<<<gx, 256, 0, st>>>((const uint32_t *)d_trk_packed, (uint32_t *)d_trk_out, d_perm + ns, ns,
                                      cfg->bsize, TRK_WORDS, (int64_t)TRK_WORDS * cfg->bsize);
  PACK_CUDA(ctx, cudaGetLastError());
  return P2Z_OK;
}

}  // extern "C"
