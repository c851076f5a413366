// p2z_step.cu -- single-layer step kernel behind p2z_step_device: the
// reference's propagateToZ (src/propagate-toz-test_OMP.cpp:623-682) and/or
// KalmanUpdate_v2 (:503-620) applied once, in place, to every track of an
// AOSOA array.  Unlike the fused hot-path kernels it makes no assumption about
// the input covariance (its z row may be non-zero), so the update here is the
// full 21-element form.  It exists for layer-by-layer parity checks and for
// callers that drive the layer loop themselves, as the reference's main does.
// It evaluates the reference's own FP32 expressions (FORM_REFERENCE) and this
// translation unit is compiled without FMA contraction.
#include <type_traits>

#include "p2z_kernels.cuh"

namespace p2z {

// Full-form KalmanUpdate_v2 on a 21-element covariance (reference :503-620).
__device__ __forceinline__ void update_v2_full(float (&p)[6], float (&C)[21], const float (&hp)[3],
                                               const float (&hc)[3]) {
  float r00 = C[0] + hc[0], r01 = C[1] + hc[1], r11 = C[2] + hc[2];
  const double det = (double)r00 * r11 - (double)r01 * r01;
  const float sc = (float)(1.0 / det);
  const float tmp = sc * r11;
  r01 *= -sc;
  r11 = sc * r00;
  r00 = tmp;
  // rows of C H^T: (C[0],C[1]) (C[1],C[2]) (C[3],C[4]) (C[6],C[7]) (C[10],C[11]) (C[15],C[16])
  const int rows[6][2] = {{0, 1}, {1, 2}, {3, 4}, {6, 7}, {10, 11}, {15, 16}};
  float K[6][2];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    K[i][0] = C[rows[i][0]] * r00 + C[rows[i][1]] * r01;
    K[i][1] = C[rows[i][0]] * r01 + C[rows[i][1]] * r11;
  }
  const float res0 = hp[0] - p[0], res1 = hp[1] - p[1];
#pragma unroll
  for (int i = 0; i < 6; ++i) p[i] = p[i] + K[i][0] * res0 + K[i][1] * res1;
  // packed (i,j), i >= j: e = K(i,:) . (C(0,j), C(1,j))
  float n[21];
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int j = 0; j <= i; ++j) {
      const int c0j = j == 0 ? 0 : j * (j + 1) / 2;      // (j,0)
      const int c1j = j <= 1 ? (j == 0 ? 1 : 2) : j * (j + 1) / 2 + 1;  // (j,1) or (1,j)
      const int ij = i * (i + 1) / 2 + j;
      n[ij] = C[ij] - (K[i][0] * C[c0j] + K[i][1] * C[c1j]);
    }
#pragma unroll
  for (int e = 0; e < 21; ++e) C[e] = n[e];
}

template <int B>
__global__ void __launch_bounds__(256) k_step(float *trk, const float *hits, int64_t nslots, int nlayer, int layer,
                                              int what, float kfact) {
  const int64_t slot = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= nslots) return;
  float *tp = const_cast<float *>(trk_lane<B>(trk, slot));
  const float *hp = hit_lane<B>(hits, slot, nlayer, layer, B);
  float p[6], C[21];
#pragma unroll
  for (int e = 0; e < 6; ++e) p[e] = tp[e * B];
#pragma unroll
  for (int e = 0; e < 21; ++e) C[e] = tp[(6 + e) * B];
  const int q = __float_as_int(tp[27 * B]);
  const float hpos[3] = {hp[0], hp[B], hp[2 * B]};
  const float hcov[3] = {hp[3 * B], hp[4 * B], hp[5 * B]};
  if (what & 1) {
    const float k = float(q) * kfact;
    Trk<float, float> s;
    s.x = p[0]; s.y = p[1]; s.z = p[2]; s.ipt = p[3]; s.phi = p[4]; s.theta = p[5];
    const Helix<float> hx = propagate_params_ref(s, hpos[2], k);
    const Jac<float> J = jacobian_ref(hx, k, s.ipt);
    propagate_cov_general(s, C, hx, J);
    p[0] = s.x; p[1] = s.y; p[2] = s.z; p[3] = s.ipt; p[4] = s.phi; p[5] = s.theta;
    C[0] = s.c00; C[1] = s.c10; C[2] = s.c11; C[3] = 0.f; C[4] = 0.f; C[5] = 0.f;
    C[6] = s.c30; C[7] = s.c31; C[8] = 0.f; C[9] = s.c33;
    C[10] = s.c40; C[11] = s.c41; C[12] = 0.f; C[13] = s.c43; C[14] = s.c44;
    C[15] = s.c50; C[16] = s.c51; C[17] = 0.f; C[18] = s.c53; C[19] = s.c54; C[20] = s.c55;
  }
  if (what & 2) update_v2_full(p, C, hpos, hcov);
#pragma unroll
  for (int e = 0; e < 6; ++e) tp[e * B] = p[e];
#pragma unroll
  for (int e = 0; e < 21; ++e) tp[(6 + e) * B] = C[e];
}

cudaError_t launch_step(int bsize, float *trk, const float *hits, int64_t nslots, int nlayer, int layer, int what,
                        float kfact, cudaStream_t st) {
  const int block = 128;
  const unsigned grid = (unsigned)((nslots + block - 1) / block);
  if (nslots <= 0) return cudaSuccess;
  switch (bsize) {
    case 8: k_step<8><<<grid, block, 0, st>>>(trk, hits, nslots, nlayer, layer, what, kfact); break;
    case 16: k_step<16><<<grid, block, 0, st>>>(trk, hits, nslots, nlayer, layer, what, kfact); break;
    case 32: k_step<32><<<grid, block, 0, st>>>(trk, hits, nslots, nlayer, layer, what, kfact); break;
    case 64: k_step<64><<<grid, block, 0, st>>>(trk, hits, nslots, nlayer, layer, what, kfact); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace p2z
