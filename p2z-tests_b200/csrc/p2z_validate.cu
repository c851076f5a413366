// p2z_validate.cu -- the reference's validation block (src/propagate-toz-test_OMP.cpp:
// 758-864) as a GPU reduction over device-resident output tracks.
//
// Per track, the values and the selection are the host block's double
// expressions (p2z_validate_partial), so the counts are identical and every
// summand is identical; only the order of the sums differs: each thread sums a
// grid-stride range, warps and blocks reduce by fixed trees, and one finishing
// block sums the per-block partials in block order.  The result is the same
// from run to run.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>

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

constexpr int kVals = 12;       // 9 sums (pass 1) or 6 squared deviations (pass 2), 3 counts
constexpr int kThreads = 256;

struct Means {
  double m[6];
};

__device__ __forceinline__ void warp_sum(double (&v)[kVals]) {
#pragma unroll
  for (int i = 0; i < kVals; ++i)
    for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_down_sync(0xffffffffu, v[i], o);
}

// Block sums of its grid-stride share of the tracks into part[blockIdx.x].
template <int B>
__global__ void __launch_bounds__(kThreads) k_validate(const float *__restrict__ trk, int64_t ntracks, double hx,
                                                        double hy, double hz, int pass2, Means mu,
                                                        double *__restrict__ part) {
  double v[kVals];
#pragma unroll
  for (int i = 0; i < kVals; ++i) v[i] = 0.0;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < ntracks;
       g += (int64_t)gridDim.x * blockDim.x) {
    // ntrks is a multiple of B, so track it of event ie is lane g % B of batch g / B
    const float *b = trk + (g / B) * (int64_t)(TRK_WORDS * B) + (g % B);
    const double x_ = b[0], y_ = b[B], z_ = b[2 * B];
    const double pt_ = 1. / (double)b[3 * B], phi_ = b[4 * B], theta_ = b[5 * B];
    if (!(isfinite(x_) && isfinite(y_) && isfinite(z_) && isfinite(pt_) && isfinite(phi_) && isfinite(theta_))) {
      v[9] += 1.0;
      continue;
    }
    if (fabs((x_ - hx) / hx) > 1. || fabs((y_ - hy) / hy) > 1. || fabs((z_ - hz) / hz) > 1. ||
        fabs((pt_ - 12.) / 12.) > 1. || fabs((phi_ - 1.3) / 1.3) > 1. || fabs((theta_ - 2.8) / 2.8) > 1.) {
      v[10] += 1.0;
      continue;
    }
    const double dx = (x_ - hx) / x_, dy = (y_ - hy) / y_, dz = (z_ - hz) / z_;
    if (!pass2) {
      v[0] += x_;
      v[1] += y_;
      v[2] += z_;
      v[3] += dx;
      v[4] += dy;
      v[5] += dz;
      v[6] += pt_;
      v[7] += phi_;
      v[8] += theta_;
    } else {
      const double d[6] = {x_ - mu.m[0], y_ - mu.m[1], z_ - mu.m[2], dx - mu.m[3], dy - mu.m[4], dz - mu.m[5]};
#pragma unroll
      for (int i = 0; i < 6; ++i) v[i] += d[i] * d[i];
    }
    v[11] += 1.0;
  }
  warp_sum(v);
  __shared__ double sh[kThreads / 32][kVals];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
    for (int i = 0; i < kVals; ++i) sh[w][i] = v[i];
  __syncthreads();
  if (threadIdx.x < kVals) {
    double s = 0.0;
    for (int k = 0; k < kThreads / 32; ++k) s += sh[k][threadIdx.x];
    part[(int64_t)blockIdx.x * kVals + threadIdx.x] = s;
  }
}

// One block: out[i] = sum over blocks of part[b][i], in block order per
// thread stripe and then a fixed tree.
__global__ void __launch_bounds__(kThreads) k_validate_finish(const double *__restrict__ part, int nblocks,
                                                               double *__restrict__ out) {
  __shared__ double sh[kThreads][kVals];
  double v[kVals];
#pragma unroll
  for (int i = 0; i < kVals; ++i) v[i] = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += kThreads)
#pragma unroll
    for (int i = 0; i < kVals; ++i) v[i] += part[(int64_t)b * kVals + i];
#pragma unroll
  for (int i = 0; i < kVals; ++i) sh[threadIdx.x][i] = v[i];
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
      for (int i = 0; i < kVals; ++i) sh[threadIdx.x][i] += sh[threadIdx.x + s][i];
    __syncthreads();
  }
  if (threadIdx.x < kVals) out[threadIdx.x] = sh[0][threadIdx.x];
}

#define VAL_CUDA(ctx, call)                                                                      \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) {                                                                     \
      char m_[300];                                                                              \
      std::snprintf(m_, sizeof m_, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__,  \
                    __LINE__);                                                                   \
      return context_fail((ctx), P2Z_CUDA_ERROR, m_);                                            \
    }                                                                                            \
  } while (0)

p2z_status pass(p2z_context *ctx, const void *d_trk, int B, int64_t nevts, int64_t ntrks, const float h[3],
                const double *means, p2z_validation_partial *acc, cudaStream_t st) {
  std::memset(acc, 0, sizeof *acc);
  const int64_t n = nevts * ntrks;
  if (n == 0) return P2Z_OK;
  int nsm = 0;
  VAL_CUDA(ctx, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, context_device(ctx)));
  const int nblocks = (int)std::min<int64_t>((int64_t)nsm * 8, (n + kThreads - 1) / kThreads);
  double *part = (double *)context_scratch(ctx, sizeof(double) * kVals * ((size_t)nblocks + 1));
  if (!part) return context_fail(ctx, P2Z_OOM, "validation scratch allocation failed");
  double *out = part + (size_t)nblocks * kVals;
  Means mu;
  for (int i = 0; i < 6; ++i) mu.m[i] = means ? means[i] : 0.0;
  const double hx = h[0], hy = h[1], hz = h[2];
  const float *t = (const float *)d_trk;
  switch (B) {
    case 8: k_validate<8><<<nblocks, kThreads, 0, st>>>(t, n, hx, hy, hz, means != nullptr, mu, part); break;
    case 16: k_validate<16><<<nblocks, kThreads, 0, st>>>(t, n, hx, hy, hz, means != nullptr, mu, part); break;
    case 32: k_validate<32><<<nblocks, kThreads, 0, st>>>(t, n, hx, hy, hz, means != nullptr, mu, part); break;
    default: k_validate<64><<<nblocks, kThreads, 0, st>>>(t, n, hx, hy, hz, means != nullptr, mu, part); break;
  }
  k_validate_finish<<<1, kThreads, 0, st>>>(part, nblocks, out);
  VAL_CUDA(ctx, cudaGetLastError());
  double r[kVals];
  VAL_CUDA(ctx, cudaMemcpyAsync(r, out, sizeof r, cudaMemcpyDeviceToHost, st));
  VAL_CUDA(ctx, cudaStreamSynchronize(st));
  if (!means)
    for (int i = 0; i < 9; ++i) acc->sum[i] = r[i];
  else
    for (int i = 0; i < 6; ++i) acc->sq[i] = r[i];
  acc->nnans = (int64_t)r[9];
  acc->nfail = (int64_t)r[10];
  acc->ngood = (int64_t)r[11];
  return P2Z_OK;
}

p2z_status check(p2z_context *ctx, const void *d_trk, int bsize, int64_t nevts, int64_t ntrks, const float *h,
                 const void *out) {
  if (!ctx) {
    set_context_free_error("context is NULL");
    return P2Z_BAD_ARG;
  }
  if (!h || !out) return context_fail(ctx, P2Z_BAD_ARG, "NULL argument");
  if (!(bsize == 8 || bsize == 16 || bsize == 32 || bsize == 64))
    return context_fail(ctx, P2Z_UNSUPPORTED, "bsize not in {8,16,32,64}");
  if (nevts < 0 || ntrks < 0 || ntrks % bsize)
    return context_fail(ctx, P2Z_BAD_ARG, "nevts/ntrks invalid (ntrks must be a multiple of bsize)");
  if (nevts * ntrks > 0 && !d_trk) return context_fail(ctx, P2Z_BAD_ARG, "NULL device buffer");
  return P2Z_OK;
}

}  // namespace

extern "C" {

p2z_status p2z_validate_partial_device(p2z_context *ctx, const void *d_trk_out, int bsize, int64_t nevts,
                                       int64_t ntrks, const float hit_last[3], const double means[6],
                                       p2z_validation_partial *acc, void *stream) {
  p2z_status r = check(ctx, d_trk_out, bsize, nevts, ntrks, hit_last, acc);
  if (r != P2Z_OK) return r;
  VAL_CUDA(ctx, cudaSetDevice(context_device(ctx)));
  return pass(ctx, d_trk_out, bsize, nevts, ntrks, hit_last, means, acc,
              stream ? (cudaStream_t)stream : context_stream(ctx));
}

p2z_status p2z_validate_device(p2z_context *ctx, const void *d_trk_out, int bsize, int64_t nevts, int64_t ntrks,
                               const float hit_last[3], p2z_validation *v, void *stream) {
  p2z_status r = check(ctx, d_trk_out, bsize, nevts, ntrks, hit_last, v);
  if (r != P2Z_OK) return r;
  VAL_CUDA(ctx, cudaSetDevice(context_device(ctx)));
  cudaStream_t st = stream ? (cudaStream_t)stream : context_stream(ctx);
  p2z_validation_partial p1, p2;
  r = pass(ctx, d_trk_out, bsize, nevts, ntrks, hit_last, nullptr, &p1, st);
  if (r != P2Z_OK) return r;
  double means[6];
  p2z_validate_means(&p1, means);
  r = pass(ctx, d_trk_out, bsize, nevts, ntrks, hit_last, means, &p2, st);
  if (r != P2Z_OK) return r;
  return p2z_validate_combine(&p1, &p2, v);
}

}  // extern "C"
