// p2z_kernels.cuh -- hot-path kernels (templates; instantiated per update kind
// in p2z_kern_*.cu).
//
// One thread owns one track slot (batch b, lane t of a bsize-wide AOSOA batch)
// and keeps the track's parameters and live covariance in registers across all
// its layers: the reference's per-layer loop (src/propagate-toz-test_OMP.cpp:
// 740-745, GPU form src/propagate-toz-test_CUDA_v4.cu:761-775) runs entirely on
// registers and the only memory traffic is one read of the track, one read of
// the 6 (v2) or 9 (3x3) hit words per present layer and one write of the track.
//
// Loads of the AOSOA arrays are coalesced: for a fixed element, consecutive
// lanes read consecutive words (a 32-lane warp reads 128 contiguous bytes when
// bsize >= 32, or 32-byte sector runs of bsize*4 bytes otherwise).  The hits of
// the next present layer are requested before the current layer is computed,
// so their latency overlaps the arithmetic.
#pragma once

#include <type_traits>

#include "p2z_math.cuh"

// Hit prefetch depth in the all-layers loop: how many layers ahead the hits
// are requested (0: at the start of each step; 1 or 2: before the step that
// precedes them, so their latency overlaps the arithmetic).
#ifndef P2Z_PREFETCH_DEPTH
#define P2Z_PREFETCH_DEPTH 1
#endif

namespace p2z {

constexpr int TRK_WORDS = 28;  // 6 par + 21 cov + 1 q
constexpr int HIT_WORDS = 9;   // 3 pos + 6 cov

// Kernel kinds
enum { KIND_FLAT = 0, KIND_PERSISTENT = 1, KIND_STAGED = 2 };
// Arithmetic of a kernel instance:
//  UPDK_V2       precise FP32 form (positions anchored at the last hit, anchored
//                direction), the reference's 2-D update, compensated 2x2
//                determinant; no FP64
//  UPDK_V2_COMP  the same with float-pair accumulators for x and y instead of
//                anchored positions
//  UPDK_3X3_F64  precise FP32 propagation; 3x3 inversion + Joseph update in FP64
//  UPDK_3X3_COMP precise FP32 propagation; 3x3 + Joseph in FP32 with compensated
//                cofactors, float-pair accumulators (FP64-free)
//  UPDK_F64      everything in FP64
//  UPDK_V2_REF   the reference's own FP32 evaluation (FORM_REFERENCE); its
//                translation unit is compiled without FMA contraction
enum { UPDK_V2 = 0, UPDK_V2_COMP = 1, UPDK_3X3_F64 = 2, UPDK_3X3_COMP = 3, UPDK_F64 = 4, UPDK_V2_REF = 5 };

template <int UPD>
struct Types {
  using T = typename std::conditional<UPD == UPDK_F64, double, float>::type;
  // x/y accumulators: anchored FP32 offsets (precise forms), float pairs
  // (V2_COMP), FP64 (F64), plain float (reference rounding).
  using A = typename std::conditional<
      UPD == UPDK_F64, double,
      typename std::conditional<UPD == UPDK_V2_REF, float,
                                typename std::conditional<UPD == UPDK_V2_COMP, DF, AP>::type>::type>::type;
  static constexpr int NH = (UPD == UPDK_3X3_F64 || UPD == UPDK_3X3_COMP) ? 9 : 6;
  // Register budget: kernels allow up to 256 threads per CTA and ask ptxas
  // for MIN_CTAS such CTAs per SM.  For the 2-D FP32 kinds, 3 caps them at 80
  // registers (24 resident warps per SM), which measured faster than the 88
  // ptxas picks unconstrained.  For the 3x3 update with its FP64 island, 2
  // caps it at 128 (16 warps instead of the 12 that 157-164 registers allow;
  // with the Joseph form evaluated a row at a time the cap spills 4 bytes):
  // 4.44 against 4.51 ms on the headline sample, 4.32 against 5.63 ms on the
  // masked uneven one (persistent).  1 leaves the count to ptxas.
  static constexpr int MIN_CTAS =
      (UPD == UPDK_V2 || UPD == UPDK_V2_COMP) ? 3 : (UPD == UPDK_3X3_F64 ? 2 : 1);
};

struct RunArgs {
  const float *__restrict__ trk;   // MPTRK[nbatches]
  const float *__restrict__ hits;  // MPHIT[nlayer * nbatches]
  float *__restrict__ out;         // MPTRK[nbatches]
  const uint32_t *__restrict__ mask;  // one word per slot, or null (all layers)
  int64_t slot_begin, slot_end;    // slots [begin, end) of this launch
  int nlayer;
  float kfact;
  unsigned int *status;            // bit 0: a det <= 0 was met; bit 1: a staging wait timed out;
                                   // bit 2: a non-finite input word (k_check_inputs)
  unsigned long long *queue;       // persistent kernels: next work item
  int64_t ws;                      // SoA layout (B == 0): slots in the arrays = word stride
  // Sorted windows (masked kernels only): the launch's slots are split into windows
  // of `win` slots from slot_begin; the thread at linear slot s processes
  // slot window_base(s) + perm[s].  perm == nullptr: s itself.
  const uint8_t *__restrict__ perm;
  int win;                         // slots per window, a power of two <= 256
  // 1: each thread first asks L2 for its batch's whole hit block (AOSOA), so
  // that a launch too small to fill the GPU -- whose warps have no others to
  // hide a layer's DRAM latency behind -- waits on L2 instead (set by the host).
  int l2_prefetch;
};

// The slot a thread processes (see RunArgs::perm).
__device__ __forceinline__ int64_t map_slot(const RunArgs &a, int64_t s) {
  if (a.perm == nullptr) return s;
  const int64_t base = a.slot_begin + ((s - a.slot_begin) & ~(int64_t)(a.win - 1));
  return base + __ldg(a.perm + s);
}

// Layouts.  B > 0: the reference's AOSOA batches of width B (element e of a
// lane at e*B from the lane's first word).  B == 0: SoA -- one batch as wide as
// the whole array of ws slots: tracks [28][ws], hits [nlayer][9][ws].
template <int B>
__device__ __forceinline__ const float *trk_lane(const float *base, int64_t slot) {
  if constexpr (B == 0) {
    return base + slot;
  } else {
    const int64_t b = slot / B;
    const int t = (int)(slot % B);
    return base + b * (int64_t)(TRK_WORDS * B) + t;
  }
}

// Hit words of slot's batch on layer l: &pos.data[t], stride B per element.
template <int B>
__device__ __forceinline__ const float *hit_lane(const float *hits, int64_t slot, int nlayer, int l, int64_t ws) {
  if constexpr (B == 0) {
    return hits + (int64_t)l * HIT_WORDS * ws + slot;
  } else {
    const int64_t b = slot / B;
    const int t = (int)(slot % B);
    return hits + (b * nlayer + l) * (int64_t)(HIT_WORDS * B) + t;
  }
}

// Requests the hit block of slot's batch into L2: its nlayer layers are
// contiguous, nlayer * 9 * B words; the batch's B lanes share the block's
// 128-byte pieces, lane t taking pieces t, t + B, ...  Every address is inside
// the block.
template <int B>
__device__ __forceinline__ void prefetch_hits_l2(const float *hits, int64_t slot, int nlayer) {
  static_assert(B > 0, "AOSOA only");
  const int64_t b = slot / B;
  const int t = (int)(slot % B);
  const int bytes = nlayer * HIT_WORDS * B * 4;
  const char *base = reinterpret_cast<const char *>(hits + b * (int64_t)nlayer * HIT_WORDS * B);
  for (int off = t * 128; off < bytes; off += B * 128) asm volatile("prefetch.global.L2 [%0];" ::"l"(base + off));
}

// Hit words a kernel needs: x, y, z, V00, V10, V11 and, for the 3-D update,
// V20, V21, V22.
template <int NH>
struct HitRegs {
  float w[NH];
};

template <int NH>
__device__ __forceinline__ void load_hit(HitRegs<NH> &h, const float *p, int64_t ws) {
  // pos[0..2] then cov[0..NH-4]; element e of the lane at p[e*ws]
#pragma unroll
  for (int e = 0; e < NH; ++e) h.w[e] = __ldg(p + e * ws);
}

// A thread's place in its track: with TPT = 2 threads per track, lanes 2i and
// 2i+1 hold the same track; j is this lane's component of the split
// covariance propagation (propagate_cov_reduced_pair) and pm the pair's lanes.
struct PairLane {
  bool j = false;
  unsigned pm = 0xffffffffu;
};

// One propagate + update step.  GENERAL: first present layer (full 21-element
// input covariance in b21).  TPT = 2 (UPDK_V2 only): the propagation of the
// covariance is split over the lane pair; everything else is evaluated by both
// lanes.  Returns true if the update met det <= 0.
template <int UPD, int SC, bool GENERAL, int TPT = 1>
__device__ __forceinline__ bool step(Trk<typename Types<UPD>::T, typename Types<UPD>::A> &s,
                                     const typename Types<UPD>::T *b21, const HitRegs<Types<UPD>::NH> &h,
                                     typename Types<UPD>::T k, typename Types<UPD>::T ik, PairLane ln = {}) {
  static_assert(TPT == 1 || (TPT == 2 && UPD == UPDK_V2), "two threads per track: UPDK_V2 only");
  using T = typename Types<UPD>::T;
  const T zout = T(h.w[2]);
  Helix<T> hx;
  Jac<T> J;
  if constexpr (UPD == UPDK_F64) {
    hx = propagate_params_f64(s, zout, k);
    J = jacobian_precise<double, GENERAL>(hx, k, s.ipt);
  } else if constexpr (UPD == UPDK_V2_REF) {
    hx = propagate_params_ref(s, zout, k);
    J = jacobian_ref(hx, k, s.ipt);
  } else {
    hx = propagate_params_precise<SC>(s, zout, k, ik);
    J = jacobian_precise<float, GENERAL>(hx, k, s.ipt);
  }
  if constexpr (GENERAL) propagate_cov_general(s, b21, hx, J);
  else if constexpr (TPT == 2) propagate_cov_reduced_pair(s, J, ln.j, ln.pm);
  else if constexpr (P2Z_PACKED_F32X2 && std::is_same<T, float>::value && UPD != UPDK_V2_REF)
    propagate_cov_reduced_packed(s, J);  // (the reference-rounding form keeps separate roundings)
  else propagate_cov_reduced(s, J);
  if constexpr (UPD == UPDK_F64) {
    const double hp[3] = {h.w[0], h.w[1], h.w[2]};
    const double hc[3] = {h.w[3], h.w[4], h.w[5]};
    return update_v2_f64(s, hp, hc);
  } else {
    const float hp[3] = {h.w[0], h.w[1], h.w[2]};
    if constexpr (UPD == UPDK_V2 || UPD == UPDK_V2_REF) {
      const float hc[3] = {h.w[3], h.w[4], h.w[5]};
      return update_v2<typename Types<UPD>::A, (UPD == UPDK_V2_REF) ? FORM_REFERENCE : FORM_PRECISE, GENERAL>(s, hp, hc);
    } else if constexpr (UPD == UPDK_V2_COMP) {
      const float hc[3] = {h.w[3], h.w[4], h.w[5]};
      return update_v2<DF, FORM_PRECISE, GENERAL>(s, hp, hc);
    } else {
      const float hv[6] = {h.w[3], h.w[4], h.w[5], h.w[6], h.w[7], h.w[8]};
      if constexpr (UPD == UPDK_3X3_F64) return update_3x3_joseph<double>(s, hp, hv);
      else return update_3x3_joseph<float>(s, hp, hv);
    }
  }
}

// Process one track slot: load, run every present layer, store.  TPT = 2: both
// lanes of the pair load the track and its hits, and lane 0 stores the result.
template <int B, int UPD, int SC, bool MASKED, int TPT = 1>
__device__ __forceinline__ void process_slot(const RunArgs &a, int64_t slot) {
  using T = typename Types<UPD>::T;
  using A = typename Types<UPD>::A;
  constexpr int NH = Types<UPD>::NH;
  const int64_t WS = (B > 0) ? (int64_t)B : a.ws;  // word stride
  const float *tin = trk_lane<B>(a.trk, slot);
  float *tout = const_cast<float *>(trk_lane<B>(a.out, slot));

  PairLane ln;
  if constexpr (TPT == 2) {
    ln.j = (threadIdx.x & 1) != 0;
    ln.pm = 3u << (threadIdx.x & 30);
  }
  const bool writer = TPT == 1 || !ln.j;
  const uint32_t all = (a.nlayer >= 32) ? 0xffffffffu : ((1u << a.nlayer) - 1u);
  uint32_t m = MASKED ? (__ldg(a.mask + slot) & all) : all;
  if constexpr (B > 0) {
    if (a.l2_prefetch && m != 0u) prefetch_hits_l2<B>(a.hits, slot, a.nlayer);
  }

  float in[TRK_WORDS];
#pragma unroll
  for (int e = 0; e < TRK_WORDS; ++e) in[e] = __ldg(tin + e * WS);

  if (m == 0u) {  // no hits (or a padding slot): the track passes through
    if (writer) {
#pragma unroll
      for (int e = 0; e < TRK_WORDS; ++e) __stcs(tout + e * WS, in[e]);
    }
    return;
  }

  const int q = __float_as_int(in[27]);
  const float kf = float(q) * a.kfact;  // reference: q*kfact in float (:627)
  const T k = T(kf);
  const T ik = T(1) / k;

  Trk<T, A> s;
  acc_set(s.x, in[0]);
  acc_set(s.y, in[1]);
  acc_set(s.phi, in[4]);
  s.z = in[2]; s.ipt = in[3]; s.theta = in[5];
  if constexpr (UPD != UPDK_F64 && UPD != UPDK_V2_REF) init_direction(s);
  T b21[21];
#pragma unroll
  for (int e = 0; e < 21; ++e) b21[e] = T(in[6 + e]);

  bool singular = false;
  HitRegs<NH> h0, h1;
  if constexpr (!MASKED && P2Z_PREFETCH_DEPTH >= 2) {
    // every layer present; three hit buffers rotate so that the hits of the
    // next two layers are in flight during a step
    const int64_t stride = HIT_WORDS * WS;
    const float *hp = hit_lane<B>(a.hits, slot, a.nlayer, 0, WS);
    const int nl = a.nlayer;
    HitRegs<NH> h2;
    load_hit<NH>(h0, hp, WS);
    if (nl > 1) load_hit<NH>(h1, hp + stride, WS);
    if (nl > 2) load_hit<NH>(h2, hp + 2 * stride, WS);
    singular |= step<UPD, SC, true, TPT>(s, b21, h0, k, ik, ln);
    int l = 1;
    for (; l + 2 < nl; l += 3) {  // layers l, l+1, l+2 are in h1, h2 and (after the load) h0
      if (l + 2 < nl) load_hit<NH>(h0, hp + (l + 2) * stride, WS);
      singular |= step<UPD, SC, false, TPT>(s, b21, h1, k, ik, ln);
      if (l + 3 < nl) load_hit<NH>(h1, hp + (l + 3) * stride, WS);
      singular |= step<UPD, SC, false, TPT>(s, b21, h2, k, ik, ln);
      if (l + 4 < nl) load_hit<NH>(h2, hp + (l + 4) * stride, WS);
      singular |= step<UPD, SC, false, TPT>(s, b21, h0, k, ik, ln);
    }
    if (l < nl) singular |= step<UPD, SC, false, TPT>(s, b21, h1, k, ik, ln);
    if (l + 1 < nl) singular |= step<UPD, SC, false, TPT>(s, b21, h2, k, ik, ln);
  } else if constexpr (!MASKED && P2Z_PREFETCH_DEPTH == 0) {
    // every layer present, one hit buffer: each layer's hits are loaded at the
    // start of its step (latency hidden by other warps only)
    const int64_t stride = HIT_WORDS * WS;
    const float *hp = hit_lane<B>(a.hits, slot, a.nlayer, 0, WS);
    load_hit<NH>(h0, hp, WS);
    singular |= step<UPD, SC, true, TPT>(s, b21, h0, k, ik, ln);
    for (int l = 1; l < a.nlayer; ++l) {
      load_hit<NH>(h0, hp + l * stride, WS);
      singular |= step<UPD, SC, false, TPT>(s, b21, h0, k, ik, ln);
    }
  } else if constexpr (!MASKED) {
    // every layer present: counted loop, hits addressed by a running pointer;
    // two hit buffers alternate so the next layer is in flight during a step
    const int64_t stride = HIT_WORDS * WS;
    const float *hp = hit_lane<B>(a.hits, slot, a.nlayer, 0, WS);
    const int nl = a.nlayer;
    load_hit<NH>(h0, hp, WS);
    if (nl > 1) load_hit<NH>(h1, hp + stride, WS);
    singular |= step<UPD, SC, true, TPT>(s, b21, h0, k, ik, ln);
    int l = 1;
    for (; l + 1 < nl; l += 2) {
      load_hit<NH>(h0, hp + (l + 1) * stride, WS);
      singular |= step<UPD, SC, false, TPT>(s, b21, h1, k, ik, ln);
      if (l + 2 < nl) load_hit<NH>(h1, hp + (l + 2) * stride, WS);
      singular |= step<UPD, SC, false, TPT>(s, b21, h0, k, ik, ln);
    }
    if (l < nl) singular |= step<UPD, SC, false, TPT>(s, b21, h1, k, ik, ln);
  } else {
    // present layers in order: lowest set bit first
    const int64_t stride = HIT_WORDS * WS;
    const float *hp = hit_lane<B>(a.hits, slot, a.nlayer, 0, WS);
    uint32_t rest = m & (m - 1u);
    load_hit<NH>(h0, hp + (__ffs(m) - 1) * stride, WS);
    if (rest) load_hit<NH>(h1, hp + (__ffs(rest) - 1) * stride, WS);
    singular |= step<UPD, SC, true, TPT>(s, b21, h0, k, ik, ln);
    while (rest) {
      rest &= rest - 1u;  // h1 holds the layer just removed from rest
      if (rest) load_hit<NH>(h0, hp + (__ffs(rest) - 1) * stride, WS);
      singular |= step<UPD, SC, false, TPT>(s, b21, h1, k, ik, ln);
      if (!rest) break;
      rest &= rest - 1u;  // h0 holds the layer just removed
      if (rest) load_hit<NH>(h1, hp + (__ffs(rest) - 1) * stride, WS);
      singular |= step<UPD, SC, false, TPT>(s, b21, h0, k, ik, ln);
    }
  }

  const float z0 = 0.0f;
  float o[TRK_WORDS];
  o[0] = tof(s.x); o[1] = tof(s.y); o[2] = float(s.z);
  o[3] = float(s.ipt); o[4] = tof(s.phi); o[5] = float(s.theta);
  float *c = o + 6;
  c[0] = float(s.c00); c[1] = float(s.c10); c[2] = float(s.c11);
  c[3] = z0; c[4] = z0; c[5] = z0;
  c[6] = float(s.c30); c[7] = float(s.c31); c[8] = z0; c[9] = float(s.c33);
  c[10] = float(s.c40); c[11] = float(s.c41); c[12] = z0; c[13] = float(s.c43); c[14] = float(s.c44);
  c[15] = float(s.c50); c[16] = float(s.c51); c[17] = z0; c[18] = float(s.c53); c[19] = float(s.c54);
  c[20] = float(s.c55);
  o[27] = in[27];
  if (writer) {
#pragma unroll
    for (int e = 0; e < TRK_WORDS; ++e) __stcs(tout + e * WS, o[e]);
    if (singular) atomicOr(a.status, 1u);
  }
}



// One launch over slots [slot_begin, slot_end), TPT threads per slot.
template <int B, int UPD, int SC, bool MASKED, int TPT = 1>
__global__ void __launch_bounds__(256, Types<UPD>::MIN_CTAS) k_flat(RunArgs a) {
  const int64_t slot = a.slot_begin + ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / TPT;
  if (slot >= a.slot_end) return;  // (both lanes of a pair together)
  process_slot<B, UPD, SC, MASKED, TPT>(a, MASKED ? map_slot(a, slot) : slot);
}

// Persistent launch: grid = resident CTAs; each warp repeatedly takes the next
// work item of 32 / TPT slots from a device counter (reset to 0 before the
// launch) until the range is exhausted.  Work items are taken in slot order,
// so concurrently running warps read neighbouring batches.
template <int B, int UPD, int SC, bool MASKED, int TPT = 1>
__global__ void __launch_bounds__(256, Types<UPD>::MIN_CTAS) k_persistent(RunArgs a) {
  constexpr int kPer = 32 / TPT;  // slots per work item
  const int lane = threadIdx.x & 31;
  const int64_t nslots = a.slot_end - a.slot_begin;
  const unsigned long long nitems = (unsigned long long)((nslots + kPer - 1) / kPer);
  for (;;) {
    unsigned long long item = 0;
    if (lane == 0) item = atomicAdd(a.queue, 1ull);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= nitems) break;
    const int64_t slot = a.slot_begin + (int64_t)item * kPer + lane / TPT;
    if (slot < a.slot_end) process_slot<B, UPD, SC, MASKED, TPT>(a, MASKED ? map_slot(a, slot) : slot);
  }
}

// ---------------------------------------------------------------------------
// Staged persistent kernel (bsize 32, AOSOA): each warp owns one 32-track
// batch at a time.  Its hit tiles -- the NH contiguous words x 32 lanes of a
// hit batch, 768 B for the 2-D updates -- stream through a ring of
// kStages shared-memory buffers filled by bulk asynchronous copies
// (cp.async.bulk, completion counted on an mbarrier per buffer), issued by
// lane 0 up to kStages layers ahead and across into the warp's next batch; the
// next batch's 3584-B track tile is copied in while the current batch runs.
// Registers hold no prefetched hits and no load of the hot loop waits on DRAM.
// Hit masks: the warp stages the union of its lanes' layers in order; a lane
// steps only on its own layers.  Every wait is bounded: on a timeout the warp
// sets status bit 1, waits (bounded) for the copies it issued and returns.
// ---------------------------------------------------------------------------
constexpr int kStages = 4;
constexpr int kStagedWaitLimit = 1 << 21;  // try_wait polls per wait

template <int UPD>
struct StagedSmem {
  static constexpr uint32_t kTrkBytes = TRK_WORDS * 32 * 4;          // 3584
  static constexpr uint32_t kHitBytes = Types<UPD>::NH * 32 * 4;     // 768 or 1152
  static constexpr uint32_t kBarOff = kTrkBytes + kStages * kHitBytes;
  static constexpr uint32_t kWarpBytes = (kBarOff + (kStages + 1) * 8 + 127) / 128 * 128;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Bounded wait for the phase with the given parity to complete.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  for (int i = 0; i < kStagedWaitLimit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// The same for a whole warp, polled in lockstep so that the warp leaves the
// loop converged; true when every lane saw the phase complete.
__device__ __forceinline__ bool mbar_wait_warp(uint64_t *bar, uint32_t parity) {
  for (int i = 0; i < kStagedWaitLimit; ++i)
    if (__all_sync(0xffffffffu, mbar_try_wait(bar, parity))) return true;
  return false;
}
// Global -> this CTA's shared memory, bytes a multiple of 16, both addresses
// 16-byte aligned; completion adds the bytes to the mbarrier's transaction count.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

template <int UPD, int SC, bool MASKED>
__global__ void __launch_bounds__(256, Types<UPD>::MIN_CTAS) k_staged(RunArgs a) {
  constexpr int B = 32;
  constexpr int NH = Types<UPD>::NH;
  using SM = StagedSmem<UPD>;
  using T = typename Types<UPD>::T;
  using A = typename Types<UPD>::A;
  extern __shared__ __align__(128) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char *wb = smem + (size_t)warp * SM::kWarpBytes;
  float *trk_s = reinterpret_cast<float *>(wb);
  float *hit_s = reinterpret_cast<float *>(wb + SM::kTrkBytes);
  uint64_t *bars = reinterpret_cast<uint64_t *>(wb + SM::kBarOff);  // [0, kStages): hits; [kStages]: track
  if (lane == 0) {
    for (int i = 0; i <= kStages; ++i) mbar_init(&bars[i], 1);
    fence_mbar_init();
  }
  __syncwarp();

  const int nl = a.nlayer;
  const uint32_t all = (nl >= 32) ? 0xffffffffu : ((1u << nl) - 1u);
  const int S = nl < kStages ? nl : kStages;  // buffers in use
  const int64_t b0 = a.slot_begin / B;
  const unsigned long long nitems = (unsigned long long)((a.slot_end - a.slot_begin) / B);
  auto grab = [&]() -> unsigned long long {
    unsigned long long it = 0;
    if (lane == 0) it = atomicAdd(a.queue, 1ull);
    return __shfl_sync(0xffffffffu, it, 0);
  };
  // lane's mask and the warp's union of layers for an item
  auto lane_mask = [&](unsigned long long it) -> uint32_t {
    if (it >= nitems) return 0u;
    return MASKED ? (__ldg(a.mask + (b0 + (int64_t)it) * B + lane) & all) : all;
  };
  auto hit_src = [&](unsigned long long it, int l) -> const float * {
    return a.hits + ((b0 + (int64_t)it) * nl + l) * (int64_t)(HIT_WORDS * B);
  };
  auto trk_src = [&](unsigned long long it) -> const float * {
    return a.trk + (b0 + (int64_t)it) * (int64_t)(TRK_WORDS * B);
  };

  unsigned long long item = grab();
  unsigned long long next = (item < nitems) ? grab() : nitems;
  uint32_t m_cur = lane_mask(item), m_next = lane_mask(next);
  uint32_t u_cur = __reduce_or_sync(0xffffffffu, m_cur), u_next = __reduce_or_sync(0xffffffffu, m_next);
  // producer state (warp-uniform): buffer of the next copy, copies in flight
  // ahead of the consumer, source (item or next) and its layers left
  int p_st = 0, ahead = 0;
  int p_sel = 0;
  uint32_t p_bits = u_cur;
  // consumer state: buffer of the next tile and its phase parity
  int c_st = 0;
  uint32_t c_par = 0;
  uint32_t tpar = 0;    // track barrier parity
  bool trk_pending = false;
  // issue hit copies while fewer than S are ahead of the consumer; the
  // bookkeeping is warp-uniform (every lane runs it), lane 0 issues
  auto produce = [&]() {
    while (ahead < S) {
      if (p_bits == 0u && p_sel == 0) {
        p_sel = 1;
        p_bits = u_next;
      }
      if (p_bits == 0u) break;
      const int l = __ffs(p_bits) - 1;
      p_bits &= p_bits - 1u;
      if (lane == 0) {
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&bars[p_st], SM::kHitBytes);
        bulk_g2s(hit_s + p_st * (NH * B), hit_src(p_sel ? next : item, l), SM::kHitBytes, &bars[p_st]);
      }
      if (++p_st == S) p_st = 0;
      ++ahead;
    }
    __syncwarp();
  };
  if (item < nitems && lane == 0) {
    mbar_arrive_expect_tx(&bars[kStages], SM::kTrkBytes);
    bulk_g2s(trk_s, trk_src(item), SM::kTrkBytes, &bars[kStages]);
  }
  trk_pending = item < nitems;
  produce();
  bool ok = true;
  while (item < nitems) {
    // the item's track tile
    ok = mbar_wait_warp(&bars[kStages], tpar);
    if (!ok) break;
    tpar ^= 1u;
    trk_pending = false;
    float *tout = a.out + (b0 + (int64_t)item) * (int64_t)(TRK_WORDS * B) + lane;
    if (m_cur == 0u) {  // no hits (or a padding slot): the track passes through
#pragma unroll
      for (int e = 0; e < TRK_WORDS; ++e) __stcs(tout + e * B, trk_s[e * B + lane]);
    }
    const int q = __float_as_int(trk_s[27 * B + lane]);
    const float kf = float(q) * a.kfact;
    const T k = T(kf);
    const T ik = T(1) / k;
    Trk<T, A> s;
    acc_set(s.x, trk_s[0 * B + lane]);
    acc_set(s.y, trk_s[1 * B + lane]);
    acc_set(s.phi, trk_s[4 * B + lane]);
    s.z = trk_s[2 * B + lane]; s.ipt = trk_s[3 * B + lane]; s.theta = trk_s[5 * B + lane];
    if constexpr (UPD != UPDK_F64 && UPD != UPDK_V2_REF) init_direction(s);
    bool singular = false, first = true;
    // the track tile stays in use until every lane with hits has run its first
    // (general) step, which reads the input covariance from it
    bool tile_busy = true;
    auto release_tile = [&]() {
      __syncwarp();
      if (next < nitems) {
        if (lane == 0) {
          fence_proxy_async_smem();
          mbar_arrive_expect_tx(&bars[kStages], SM::kTrkBytes);
          bulk_g2s(trk_s, trk_src(next), SM::kTrkBytes, &bars[kStages]);
        }
        trk_pending = true;
      }
      tile_busy = false;
    };
    // the next staged hit tile into registers, then refill its buffer
    auto take_hit = [&](HitRegs<NH> &h) -> bool {
      if (!mbar_wait_warp(&bars[c_st], c_par)) return false;
#pragma unroll
      for (int e = 0; e < NH; ++e) h.w[e] = hit_s[c_st * (NH * B) + e * B + lane];
      __syncwarp();
      if (++c_st == S) {
        c_st = 0;
        c_par ^= 1u;
      }
      --ahead;
      produce();
      return true;
    };
    auto first_step = [&](const HitRegs<NH> &h) {
      T b21[21];
#pragma unroll
      for (int e = 0; e < 21; ++e) b21[e] = T(trk_s[(6 + e) * B + lane]);
      singular |= step<UPD, SC, true>(s, b21, h, k, ik);
      first = false;
    };
    if constexpr (!MASKED) {
      // every lane has every layer: the first is general, the rest reduced
      HitRegs<NH> h;
      ok = take_hit(h);
      if (!ok) break;
      first_step(h);
      release_tile();
      for (int l = 1; l < nl; ++l) {
        ok = take_hit(h);
        if (!ok) break;
        singular |= step<UPD, SC, false>(s, nullptr, h, k, ik);
      }
    } else {
      uint32_t ucur = u_cur;
      while (ucur) {
        const int l = __ffs(ucur) - 1;
        ucur &= ucur - 1u;
        HitRegs<NH> h;
        ok = take_hit(h);
        if (!ok) break;
        if ((m_cur >> l) & 1u) {
          if (first) first_step(h);
          else singular |= step<UPD, SC, false>(s, nullptr, h, k, ik);
        }
        if (tile_busy && __all_sync(0xffffffffu, !first || (m_cur >> l) == 0u)) release_tile();
      }
    }
    if (!ok) break;
    if (tile_busy) release_tile();
    if (!first) {
      const float z0 = 0.0f;
      float o[TRK_WORDS];
      o[0] = tof(s.x); o[1] = tof(s.y); o[2] = float(s.z);
      o[3] = float(s.ipt); o[4] = tof(s.phi); o[5] = float(s.theta);
      float *c = o + 6;
      c[0] = float(s.c00); c[1] = float(s.c10); c[2] = float(s.c11);
      c[3] = z0; c[4] = z0; c[5] = z0;
      c[6] = float(s.c30); c[7] = float(s.c31); c[8] = z0; c[9] = float(s.c33);
      c[10] = float(s.c40); c[11] = float(s.c41); c[12] = z0; c[13] = float(s.c43); c[14] = float(s.c44);
      c[15] = float(s.c50); c[16] = float(s.c51); c[17] = z0; c[18] = float(s.c53); c[19] = float(s.c54);
      c[20] = float(s.c55);
      o[27] = __int_as_float(q);
#pragma unroll
      for (int e = 0; e < TRK_WORDS; ++e) __stcs(tout + e * B, o[e]);
    }
    if (singular) atomicOr(a.status, 1u);
    // advance: the producer's "next" becomes its "item"
    item = next;
    m_cur = m_next;
    u_cur = u_next;
    next = (item < nitems) ? grab() : nitems;
    m_next = lane_mask(next);
    u_next = __reduce_or_sync(0xffffffffu, m_next);
    if (p_sel == 1) {
      p_sel = 0;
    } else {  // the producer had not reached the new item yet
      p_bits = u_cur;
    }
    produce();
  }
  if (!ok) {
    // a wait ran out: report it, then wait (bounded) for the copies this warp issued
    if (lane == 0) {
      atomicOr(a.status, 2u);
      int st = c_st;
      uint32_t par = c_par;
      for (int j = 0; j < ahead; ++j) {
        mbar_wait(&bars[st], par);
        if (++st == S) {
          st = 0;
          par ^= 1u;
        }
      }
      if (trk_pending) mbar_wait(&bars[kStages], tpar);
    }
    __syncwarp();
  }
}

// Launch description used by the dispatch functions.
struct LaunchSpec {
  RunArgs args;
  int bsize;
  bool soa;      // SoA layout (args.ws = slots in the arrays)
  int upd;       // UPDK_*
  int sc;        // SC_*
  bool masked;
  int kind;      // KIND_*
  int block;     // threads per CTA
  int grid;      // CTAs (persistent); flat computes its own
  int tpt;       // threads per track: 1, or 2 (UPDK_V2, flat and persistent kinds)
};

// P2Z_FLAG_CHECK_INPUTS (p2z_check.cu): sets status bit 2 when a word the
// pass over slots [a.slot_begin, a.slot_end) reads is NaN or Inf; B = 0: SoA
// (word stride a.ws); nh hit words per present layer.
cudaError_t launch_check_inputs(const RunArgs &a, int B, int nh, cudaStream_t st);

// Per-update-kind dispatchers (one translation unit each).
cudaError_t launch_v2(const LaunchSpec &s, cudaStream_t st);
cudaError_t launch_v2_comp(const LaunchSpec &s, cudaStream_t st);
cudaError_t launch_3x3_f64(const LaunchSpec &s, cudaStream_t st);
cudaError_t launch_3x3_comp(const LaunchSpec &s, cudaStream_t st);
cudaError_t launch_f64(const LaunchSpec &s, cudaStream_t st);
cudaError_t launch_v2_ref(const LaunchSpec &s, cudaStream_t st);
// Occupancy (resident CTAs per SM) of the kernel a spec selects.
int occupancy_v2(const LaunchSpec &s);
int occupancy_v2_comp(const LaunchSpec &s);
int occupancy_3x3_f64(const LaunchSpec &s);
int occupancy_3x3_comp(const LaunchSpec &s);
int occupancy_f64(const LaunchSpec &s);
int occupancy_v2_ref(const LaunchSpec &s);

// Shared dispatch body: picks the template instance for (B, SC, MASKED, KIND,
// threads per track).
template <int UPD, bool HAS_FAST>
struct Dispatch {
  static constexpr bool HAS_PAIR = UPD == UPDK_V2;
  template <int B, int SC, bool M>
  static const void *fn(int kind, int tpt) {
    if (kind == KIND_STAGED) {
      if constexpr (B == 32) return tpt == 1 ? (const void *)k_staged<UPD, SC, M> : nullptr;
      else return nullptr;
    }
    if (tpt == 2) {
      if constexpr (HAS_PAIR)
        return kind == KIND_PERSISTENT ? (const void *)k_persistent<B, UPD, SC, M, 2>
                                       : (const void *)k_flat<B, UPD, SC, M, 2>;
      else return nullptr;
    }
    if (tpt != 1) return nullptr;
    return kind == KIND_PERSISTENT ? (const void *)k_persistent<B, UPD, SC, M> : (const void *)k_flat<B, UPD, SC, M>;
  }
  // dynamic shared memory of a launch
  static size_t smem_bytes(const LaunchSpec &s) {
    return s.kind == KIND_STAGED ? (size_t)(s.block / 32) * StagedSmem<UPD>::kWarpBytes : 0;
  }
  template <int B, int SC>
  static const void *fn_m(bool masked, int kind, int tpt) {
    return masked ? fn<B, SC, true>(kind, tpt) : fn<B, SC, false>(kind, tpt);
  }
  template <int B>
  static const void *fn_sc(int sc, bool masked, int kind, int tpt) {
    if constexpr (HAS_FAST) {
      if (sc == SC_FAST) return fn_m<B, SC_FAST>(masked, kind, tpt);
    }
    return fn_m<B, SC_ACCURATE>(masked, kind, tpt);
  }
  static const void *select(const LaunchSpec &s) {
    if (s.soa) return fn_sc<0>(s.sc, s.masked, s.kind, s.tpt);
    switch (s.bsize) {
      case 8: return fn_sc<8>(s.sc, s.masked, s.kind, s.tpt);
      case 16: return fn_sc<16>(s.sc, s.masked, s.kind, s.tpt);
      case 32: return fn_sc<32>(s.sc, s.masked, s.kind, s.tpt);
      case 64: return fn_sc<64>(s.sc, s.masked, s.kind, s.tpt);
      default: return nullptr;
    }
  }
  static cudaError_t launch(const LaunchSpec &s, cudaStream_t st) {
    const void *f = select(s);
    if (!f) return cudaErrorInvalidValue;
    const int64_t n = s.args.slot_end - s.args.slot_begin;
    if (n <= 0) return cudaSuccess;
    int grid;
    if (s.kind == KIND_PERSISTENT || s.kind == KIND_STAGED) {
      grid = s.grid;
    } else {
      grid = (int)((n * s.tpt + s.block - 1) / s.block);
    }
    const size_t smem = smem_bytes(s);
    if (smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
    }
    RunArgs a = s.args;
    void *params[] = {&a};
    return cudaLaunchKernel(f, dim3(grid), dim3(s.block), params, smem, st);
  }
  static int occupancy(const LaunchSpec &s) {
    const void *f = select(s);
    int nb = 0;
    const size_t smem = smem_bytes(s);
    if (!f) return 0;
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, f, s.block, smem) != cudaSuccess) return 0;
    return nb;
  }
};

}  // namespace p2z
