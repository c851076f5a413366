// p2z_peak.cu -- measured denominators for the roofline fractions the
// benchmark reports (no counterpart in the reference): the FP32 fused
// multiply-add throughput of the GPU, as scalar FFMA and as the paired
// FP32x2 form, and the pinned host<->device copy rates the end-to-end path
// is bound by.  Nothing here changes a GPU setting; the clocks are whatever
// the GPU runs at.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>

#include "p2z.h"

namespace p2z {
void set_context_free_error(const char *msg);
}

namespace {

constexpr int kChains = 16;  // independent FP32 lanes of work per thread and iteration

// Every thread runs kChains independent fused multiply-add recurrences
// a <- a*m + c (|m| < 1, so they stay bounded), as kChains scalar FFMA or as
// kChains/2 paired FFMA2, for `iters` iterations: 2*kChains flops per
// iteration either way.  The result is written only if it equals a value the
// recurrences never reach, so the arithmetic cannot be removed.
template <bool PAIRED>
__global__ void __launch_bounds__(256) k_fma_peak(float *sink, int iters, float m) {
  const float c = 1e-7f * (threadIdx.x + 1);
  float total = 0.f;
  if constexpr (PAIRED) {
    float2 a[kChains / 2];
#pragma unroll
    for (int k = 0; k < kChains / 2; ++k) a[k] = make_float2(threadIdx.x * 1e-3f + k, k * 0.5f);
    const float2 mm = make_float2(m, m), cc = make_float2(c, 2.f * c);
#pragma unroll 8
    for (int i = 0; i < iters; ++i) {
#pragma unroll
      for (int k = 0; k < kChains / 2; ++k) a[k] = __ffma2_rn(a[k], mm, cc);
    }
#pragma unroll
    for (int k = 0; k < kChains / 2; ++k) total += a[k].x + a[k].y;
  } else {
    float a[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = threadIdx.x * 1e-3f + k;
#pragma unroll 8
    for (int i = 0; i < iters; ++i) {
#pragma unroll
      for (int k = 0; k < kChains; ++k) a[k] = fmaf(a[k], m, c);
    }
#pragma unroll
    for (int k = 0; k < kChains; ++k) total += a[k];
  }
  if (total == -1234.5f) sink[blockIdx.x * blockDim.x + threadIdx.x] = total;
}

struct Scoped {
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  float *sink = nullptr;
  void *dev = nullptr, *host = nullptr, *dev2 = nullptr, *host2 = nullptr;
  cudaStream_t st2 = nullptr;
  ~Scoped() {
    if (st) cudaStreamSynchronize(st);
    if (st2) cudaStreamSynchronize(st2);
    if (sink) cudaFree(sink);
    if (dev) cudaFree(dev);
    if (dev2) cudaFree(dev2);
    if (host) cudaFreeHost(host);
    if (host2) cudaFreeHost(host2);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    if (st2) cudaStreamDestroy(st2);
  }
};

p2z_status cuda_fail(const char *what, cudaError_t e) {
  char buf[256];
  std::snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
  cudaGetLastError();
  p2z::set_context_free_error(buf);
  return e == cudaErrorMemoryAllocation ? P2Z_OOM : P2Z_CUDA_ERROR;
}

#define PK_CUDA(call)                              \
  do {                                             \
    cudaError_t e_ = (call);                       \
    if (e_ != cudaSuccess) return cuda_fail(#call, e_); \
  } while (0)

}  // namespace

extern "C" p2z_status p2z_measure_peaks(int device, size_t copy_bytes, int reps, p2z_peaks *out) {
  if (!out) {
    p2z::set_context_free_error("p2z_measure_peaks: out is NULL");
    return P2Z_BAD_ARG;
  }
  std::memset(out, 0, sizeof *out);
  if (reps <= 0) reps = 5;
  if (copy_bytes == 0) copy_bytes = (size_t)1 << 30;
  copy_bytes = (copy_bytes + 4095) & ~(size_t)4095;
  if (device >= 0) PK_CUDA(cudaSetDevice(device));
  int dev = 0, sms = 0;
  PK_CUDA(cudaGetDevice(&dev));
  PK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  Scoped s;
  PK_CUDA(cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking));
  PK_CUDA(cudaStreamCreateWithFlags(&s.st2, cudaStreamNonBlocking));
  PK_CUDA(cudaEventCreate(&s.e0));
  PK_CUDA(cudaEventCreate(&s.e1));
  // FP32: 8 CTAs of 256 threads per SM (64 warps, the SM's limit), about 10 ms per launch
  const int threads = 256, blocks = sms * 8, iters = 65536;
  PK_CUDA(cudaMalloc(&s.sink, sizeof(float) * (size_t)blocks * threads));
  const double flops = 2.0 * kChains * (double)iters * blocks * threads;
  for (int paired = 0; paired < 2; ++paired) {
    double best = 1e30;
    for (int r = 0; r <= reps; ++r) {  // the first launch is a warm-up
      PK_CUDA(cudaEventRecord(s.e0, s.st));
      if (paired) k_fma_peak<true><<<blocks, threads, 0, s.st>>>(s.sink, iters, 0.999f);
      else k_fma_peak<false><<<blocks, threads, 0, s.st>>>(s.sink, iters, 0.999f);
      PK_CUDA(cudaGetLastError());
      PK_CUDA(cudaEventRecord(s.e1, s.st));
      PK_CUDA(cudaEventSynchronize(s.e1));
      float ms = 0.f;
      PK_CUDA(cudaEventElapsedTime(&ms, s.e0, s.e1));
      if (r > 0) best = std::min(best, (double)ms);
    }
    (paired ? out->fp32_ffma2_tflops : out->fp32_ffma_tflops) = flops / (best * 1e-3) / 1e12;
  }
  // pinned copies, one large cudaMemcpyAsync each way, then both at once on two streams
  PK_CUDA(cudaMalloc(&s.dev, copy_bytes));
  PK_CUDA(cudaMalloc(&s.dev2, copy_bytes));
  PK_CUDA(cudaHostAlloc(&s.host, copy_bytes, cudaHostAllocPortable));
  PK_CUDA(cudaHostAlloc(&s.host2, copy_bytes, cudaHostAllocPortable));
  std::memset(s.host, 1, copy_bytes);
  std::memset(s.host2, 2, copy_bytes);
  for (int dir = 0; dir < 3; ++dir) {
    double best = 1e30;
    for (int r = 0; r <= reps; ++r) {
      PK_CUDA(cudaEventRecord(s.e0, s.st));
      if (dir == 0 || dir == 2) PK_CUDA(cudaMemcpyAsync(s.dev, s.host, copy_bytes, cudaMemcpyHostToDevice, s.st));
      if (dir == 1) PK_CUDA(cudaMemcpyAsync(s.host2, s.dev2, copy_bytes, cudaMemcpyDeviceToHost, s.st));
      if (dir == 2) {
        PK_CUDA(cudaStreamWaitEvent(s.st2, s.e0, 0));
        PK_CUDA(cudaMemcpyAsync(s.host2, s.dev2, copy_bytes, cudaMemcpyDeviceToHost, s.st2));
        cudaEvent_t j = nullptr;
        PK_CUDA(cudaEventCreateWithFlags(&j, cudaEventDisableTiming));
        cudaEventRecord(j, s.st2);
        cudaStreamWaitEvent(s.st, j, 0);
        cudaEventDestroy(j);
      }
      PK_CUDA(cudaEventRecord(s.e1, s.st));
      PK_CUDA(cudaEventSynchronize(s.e1));
      float ms = 0.f;
      PK_CUDA(cudaEventElapsedTime(&ms, s.e0, s.e1));
      if (r > 0) best = std::min(best, (double)ms);
    }
    const double gbs = (dir == 2 ? 2.0 : 1.0) * (double)copy_bytes / (best * 1e-3) / 1e9;
    if (dir == 0) out->h2d_gbs = gbs;
    else if (dir == 1) out->d2h_gbs = gbs;
    else out->bidir_gbs = gbs;
  }
  out->copy_bytes = (int64_t)copy_bytes;
  out->sms = sms;
  return P2Z_OK;
}
