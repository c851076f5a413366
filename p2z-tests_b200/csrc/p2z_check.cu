// p2z_check.cu -- P2Z_FLAG_CHECK_INPUTS: a scan of the input words a pass
// reads for NaN and Inf before the pass.
//
// Per slot with at least one present layer (mask word != 0; every slot of a
// uniform run): the 27 floating-point track words (6 parameters, 21
// covariance elements; q is an integer) and, on every present layer, the hit
// words the update kind reads (x, y, z, V00, V10, V11 for the 2-D updates; all
// 9 for the 3-D ones).  Padding slots and absent layers are not read by the
// pass and are not scanned.  A non-finite word sets bit 2 of the status word.
// No counterpart in the reference, which counts NaN outputs in its validation
// block only (src/propagate-toz-test_OMP.cpp:750-876).
#include <cuda_runtime.h>

#include "p2z_kernels.cuh"

namespace p2z {

constexpr unsigned kStatusNonfinite = 4u;

template <int B>
__global__ void __launch_bounds__(256) k_check_inputs(RunArgs a, int nh) {
  const int64_t s = a.slot_begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.slot_end) return;
  const int64_t WS = (B > 0) ? (int64_t)B : a.ws;
  const uint32_t all = (a.nlayer >= 32) ? 0xffffffffu : ((1u << a.nlayer) - 1u);
  uint32_t m = a.mask ? (__ldg(a.mask + s) & all) : all;
  if (m == 0u) return;
  bool ok = true;
  const float *t = trk_lane<B>(a.trk, s);
  for (int e = 0; e < TRK_WORDS - 1; ++e) ok &= isfinite(__ldg(t + e * WS));
  while (m) {
    const int l = __ffs(m) - 1;
    m &= m - 1u;
    const float *h = hit_lane<B>(a.hits, s, a.nlayer, l, WS);
    for (int e = 0; e < nh; ++e) ok &= isfinite(__ldg(h + e * WS));
  }
  if (!ok) atomicOr(a.status, kStatusNonfinite);
}

// Slots [a.slot_begin, a.slot_end) of a pass with batch width B (0: SoA) and
// nh hit words read per present layer.
cudaError_t launch_check_inputs(const RunArgs &a, int B, int nh, cudaStream_t st) {
  const int64_t n = a.slot_end - a.slot_begin;
  if (n <= 0) return cudaSuccess;
  const unsigned grid = (unsigned)((n + 255) / 256);
  switch (B) {
    case 0: k_check_inputs<0><<<grid, 256, 0, st>>>(a, nh); break;
    case 8: k_check_inputs<8><<<grid, 256, 0, st>>>(a, nh); break;
    case 16: k_check_inputs<16><<<grid, 256, 0, st>>>(a, nh); break;
    case 32: k_check_inputs<32><<<grid, 256, 0, st>>>(a, nh); break;
    case 64: k_check_inputs<64><<<grid, 256, 0, st>>>(a, nh); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace p2z
