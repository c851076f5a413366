// p2z_noalloc.cu -- p2z_run_device_noalloc: the persistent work-queue pass
// on device buffers without allocating anything.
//
// Who needs it: applications whose device memory belongs to another allocator
// that must see every byte (a framework's caching allocator, an experiment's
// memory manager with fixed budgets), and latency-critical processing paths on
// which cudaMalloc and cudaFree are not allowed because they can synchronise
// the whole device.  The regular entry points keep their scratch in a
// p2z_context, whose creation calls cudaMalloc.
//
// The persistent kernel needs scratch global memory beyond its inputs and
// outputs: a work counter, a status word and -- for uneven events passed
// without a hit mask -- one padding-mask word per track slot plus the events'
// slot offsets.  Here that scratch is the file-scope array g_noalloc_scratch,
// of fixed size, which every GPU that loads this library holds until the
// process exits.  Host code must not use the array's name as a device
// address: it is a host-side stand-in.  The device address is obtained once
// per device with cudaGetSymbolAddress, with that device current, on the
// first call on that device, and kept for the life of the process (a device
// reset, which reloads the library's module at a new address, makes it stale).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "p2z.h"
#include "p2z_kernels.cuh"

namespace p2z {
void set_context_free_error(const char *msg);  // p2z_api.cu
}

using namespace p2z;

namespace {

// Scratch layout (byte offsets):
//   [0, 8)        persistent work counter (zeroed by every call)
//   [8, 12)       status word (zeroed by every call)
//   [256, ...)    event track counts, int64[P2Z_NOALLOC_MAX_EVENTS]
//   then          event first-slot offsets, int64[P2Z_NOALLOC_MAX_EVENTS + 1]
//   then          padding masks, uint32[P2Z_NOALLOC_MAX_SLOTS]
constexpr size_t kCounts = 256;
constexpr size_t kOffsets = kCounts + sizeof(int64_t) * P2Z_NOALLOC_MAX_EVENTS;
constexpr size_t kMasks = kOffsets + sizeof(int64_t) * (P2Z_NOALLOC_MAX_EVENTS + 1);
constexpr size_t kScratchBytes = kMasks + sizeof(uint32_t) * P2Z_NOALLOC_MAX_SLOTS;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
void *g_scratch_addr[64];  // device address of g_noalloc_scratch, per device

// Errors are reported through p2z_last_error(NULL), like other context-free failures.
p2z_status fail(p2z_status st, const char *msg) {
  p2z::set_context_free_error(msg);
  return st;
}

// Exclusive prefix sum of the events' slot counts (ceil(n/B)*B) into the
// offsets array: one block of 1024 threads, each owning a contiguous chunk.
__global__ void k_event_offsets(int nevts, int B) {
  __shared__ int64_t part[1024];
  const int64_t *counts = reinterpret_cast<const int64_t *>(g_noalloc_scratch + kCounts);
  int64_t *offs = reinterpret_cast<int64_t *>(g_noalloc_scratch + kOffsets);
  const int t = threadIdx.x;
  const int chunk = (nevts + 1023) / 1024;
  const int e0 = min(nevts, t * chunk), e1 = min(nevts, e0 + chunk);
  int64_t sum = 0;
  for (int e = e0; e < e1; ++e) sum += ((counts[e] + B - 1) / B) * B;
  part[t] = sum;
  __syncthreads();
  for (int d = 1; d < 1024; d <<= 1) {  // inclusive scan of the chunk sums
    const int64_t v = (t >= d) ? part[t - d] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int64_t run = part[t] - sum;  // exclusive start of this chunk
  for (int e = e0; e < e1; ++e) {
    offs[e] = run;
    run += ((counts[e] + B - 1) / B) * B;
  }
  if (t == 1023) offs[nevts] = part[1023];
}

// Padding mask: every layer for a real track, 0 for the padding lanes that
// round each event up to whole batches.
__global__ void k_padding_mask(int nevts, int64_t nslots, uint32_t all) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslots) return;
  const int64_t *counts = reinterpret_cast<const int64_t *>(g_noalloc_scratch + kCounts);
  const int64_t *offs = reinterpret_cast<const int64_t *>(g_noalloc_scratch + kOffsets);
  uint32_t *mask = reinterpret_cast<uint32_t *>(g_noalloc_scratch + kMasks);
  int lo = 0, hi = nevts;  // last event with offs[e] <= s
  while (hi - lo > 1) {
    const int mid = (lo + hi) / 2;
    if (offs[mid] <= s) lo = mid;
    else hi = mid;
  }
  mask[s] = (s - offs[lo] < counts[lo]) ? all : 0u;
}

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

}  // namespace

extern "C" p2z_status p2z_run_device_noalloc(const p2z_config *cfg, const void *d_trk_in, const void *d_hits,
                                             const uint32_t *d_hit_mask, void *d_trk_out, void *stream) {
  if (!cfg) return fail(P2Z_BAD_ARG, "config is NULL");
  if (cfg->abi_version != P2Z_ABI_VERSION) return fail(P2Z_BAD_ARG, "abi_version mismatch");
  const int B = cfg->bsize;
  if (!(B == 8 || B == 16 || B == 32 || B == 64)) return fail(P2Z_UNSUPPORTED, "bsize not in {8,16,32,64}");
  if (cfg->layout != P2Z_LAYOUT_AOSOA) return fail(P2Z_UNSUPPORTED, "only the AOSOA layout is supported here");
  if (cfg->nlayer < 1 || cfg->nlayer > 32) return fail(P2Z_BAD_ARG, "nlayer not in 1..32");
  if (cfg->nevts < 0) return fail(P2Z_BAD_ARG, "nevts < 0");
  if (cfg->niter < 0) return fail(P2Z_BAD_ARG, "niter < 0");
  if (!std::isfinite(cfg->kfact)) return fail(P2Z_BAD_ARG, "kfact is not finite");
  if (cfg->update < P2Z_UPDATE_V2 || cfg->update > P2Z_UPDATE_F64) return fail(P2Z_BAD_ARG, "unknown update kind");
  if ((cfg->flags & P2Z_FLAG_REFERENCE_ROUNDING) && cfg->update != P2Z_UPDATE_V2)
    return fail(P2Z_UNSUPPORTED, "P2Z_FLAG_REFERENCE_ROUNDING applies to P2Z_UPDATE_V2 only");
  if (cfg->block_threads != 0 && (cfg->block_threads < 32 || cfg->block_threads > 256 || cfg->block_threads % 32))
    return fail(P2Z_BAD_ARG, "block_threads not a multiple of 32 in 32..256");
  if (cfg->flags & ~(uint32_t)(P2Z_FLAG_CHECK_INPUTS | P2Z_FLAG_STRICT | P2Z_FLAG_NO_GRAPH | P2Z_FLAG_ACCURATE_TRIG |
                               P2Z_FLAG_FULL_HITS | P2Z_FLAG_REFERENCE_ROUNDING | P2Z_FLAG_PER_EVENT_STREAMS |
                               P2Z_FLAG_SORT_WINDOWS))
    return fail(P2Z_BAD_ARG, "unknown flag bits");
  // The status word lives in the shared scratch and no call returns it, so
  // the flags that report through it are refused rather than ignored.
  if (cfg->flags & (P2Z_FLAG_STRICT | P2Z_FLAG_CHECK_INPUTS))
    return fail(P2Z_UNSUPPORTED, "P2Z_FLAG_STRICT and P2Z_FLAG_CHECK_INPUTS need p2z_run_device (this entry point "
                                 "returns no status from the device)");
  // slots of the run, without allocating: sum over events of ceil(n/B)*B
  const bool uneven = cfg->event_ntrks != nullptr;
  int64_t nslots = 0;
  if (uneven) {
    for (int64_t e = 0; e < cfg->nevts; ++e) {
      if (cfg->event_ntrks[e] < 0) return fail(P2Z_BAD_ARG, "negative event track count");
      nslots += ((cfg->event_ntrks[e] + B - 1) / B) * B;
    }
  } else {
    if (cfg->ntrks < 0 || cfg->ntrks % B) return fail(P2Z_BAD_ARG, "ntrks is not a multiple of bsize");
    nslots = cfg->nevts * cfg->ntrks;
  }
  const bool build_mask = uneven && d_hit_mask == nullptr;
  if (build_mask && (cfg->nevts > P2Z_NOALLOC_MAX_EVENTS || nslots > P2Z_NOALLOC_MAX_SLOTS)) {
    char msg[200];
    std::snprintf(msg, sizeof msg,
                  "uneven run without a hit mask needs %lld slots and %lld events of scratch; "
                  "the limits are %d slots and %d events (pass a hit mask or use p2z_run_device)",
                  (long long)nslots, (long long)cfg->nevts, P2Z_NOALLOC_MAX_SLOTS, P2Z_NOALLOC_MAX_EVENTS);
    return fail(P2Z_BAD_ARG, msg);
  }
  if (nslots > 0 && (!d_trk_in || !d_hits || !d_trk_out)) return fail(P2Z_BAD_ARG, "NULL device buffer");
  if (nslots > 0 && d_trk_in == d_trk_out) return fail(P2Z_BAD_ARG, "d_trk_out must not alias d_trk_in");

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64) return fail(P2Z_NO_DEVICE, "no current CUDA device");
  unsigned char *scratch;
  {
    // once per device, with that device current: the array's device address
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
      void *ptr = nullptr;
      e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(P2Z_CUDA_ERROR, "cudaGetSymbolAddress of the scratch array failed");
      }
      g_scratch_addr[dev] = ptr;
    }
    scratch = static_cast<unsigned char *>(g_scratch_addr[dev]);
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const uint32_t all = cfg->nlayer >= 32 ? 0xffffffffu : ((1u << cfg->nlayer) - 1u);
  if (nslots == 0) return P2Z_OK;
  const uint32_t *mask = d_hit_mask;
  if (build_mask) {
    if ((e = cudaMemcpyAsync(scratch + kCounts, cfg->event_ntrks, sizeof(int64_t) * cfg->nevts,
                             cudaMemcpyHostToDevice, st)) != cudaSuccess)
      return fail(P2Z_CUDA_ERROR, cudaGetErrorString(e));
    k_event_offsets<<<1, 1024, 0, st>>>((int)cfg->nevts, B);
    k_padding_mask<<<(unsigned)((nslots + 255) / 256), 256, 0, st>>>((int)cfg->nevts, nslots, all);
    mask = reinterpret_cast<const uint32_t *>(scratch + kMasks);
  }
  LaunchSpec spec;
  std::memset(&spec, 0, sizeof spec);
  spec.tpt = 1;
  spec.args.trk = static_cast<const float *>(d_trk_in);
  spec.args.hits = static_cast<const float *>(d_hits);
  spec.args.out = static_cast<float *>(d_trk_out);
  spec.args.mask = mask;
  spec.args.slot_begin = 0;
  spec.args.slot_end = nslots;
  spec.args.nlayer = cfg->nlayer;
  spec.args.kfact = cfg->kfact != 0.f ? cfg->kfact : (float)(100. / (-0.299792458 * 3.8112));
  spec.args.queue = reinterpret_cast<unsigned long long *>(scratch);
  spec.args.status = reinterpret_cast<unsigned int *>(scratch + 8);
  spec.bsize = B;
  spec.upd = (cfg->flags & P2Z_FLAG_REFERENCE_ROUNDING) ? UPDK_V2_REF : cfg->update;
  spec.sc = (cfg->flags & P2Z_FLAG_ACCURATE_TRIG) ? SC_ACCURATE : SC_FAST;
  spec.masked = mask != nullptr;
  spec.kind = KIND_PERSISTENT;
  spec.block = cfg->block_threads ? cfg->block_threads : 128;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int occ = std::max(1, kernel_occupancy(spec));
  const int64_t items = (nslots + 31) / 32;
  spec.grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)occ * nsm, (items * 32 + spec.block - 1) / spec.block));
  const int niter = cfg->niter > 0 ? cfg->niter : 1;
  for (int it = 0; it < niter; ++it) {
    // what must start at zero: the work counter and the status word
    if ((e = cudaMemsetAsync(scratch, 0, 16, st)) != cudaSuccess) return fail(P2Z_CUDA_ERROR, cudaGetErrorString(e));
    if ((e = dispatch_kernel(spec, st)) != cudaSuccess) return fail(P2Z_CUDA_ERROR, cudaGetErrorString(e));
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(P2Z_CUDA_ERROR, cudaGetErrorString(e));
  return P2Z_OK;
}
