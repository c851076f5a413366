// p2z_prep.cu -- p2z_prepare_device: the reference's input preparation
// (srand(1), prepareTracks, prepareHits: src/propagate-toz-test_OMP.cpp:
// 127-145, :243-293) generated on the GPU into device buffers, word for word
// the output of p2z_prepare.
//
// The reference draws every smearing factor from one sequential stream: the C
// library's rand(), turned into N(0,1) variates by the polar method, two per
// accepted attempt.  That stream parallelises:
//  * rand() is an additive lagged Fibonacci generator (r[k] = r[k-31] +
//    r[k-3] mod 2^32, output r[k] >> 1; p2z_refrng.h), linear over Z/2^32, so
//    the 31-word state D draws ahead is a 31x31 matrix power times the state.
//    The host computes the state at the start of every chunk of kDraws draws
//    (one matrix-vector product per chunk).
//  * attempt j of the polar method always consumes draws 2j and 2j+1, and
//    whether it is accepted depends on those two draws only.  A first kernel
//    counts each chunk's accepted attempts; their prefix sum gives each
//    chunk's first accepted-attempt index, and accepted attempt a yields
//    variates 2a and 2a+1 (randn returns the second variate of a pair on the
//    next call).
//  * variate v is the smearing factor of one output word: the first
//    nevts*ntrks*27 are prepareTracks' (track order, then element), the rest
//    prepareHits' (layer, event, batch, lane, element).
// A second kernel regenerates each chunk and writes every variate's word.
// The arithmetic is the host's (p2z_host.cpp, p2z_refrng.h) with one
// exception: the variate's log is (float)log((double)W), correctly rounded,
// where the host calls the C library's logf, which differs by one unit in
// the last place for about 0.3% of the variates; on 200M variates that
// changed no output word (the smearing factor 1 + smear*r rounds the same),
// and the GPU tests compare the two outputs word for word.  This translation
// unit is compiled without FMA contraction, as the host side is.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "p2z.h"
#include "p2z_refrng.h"

namespace p2z {
int context_device(const p2z_context *ctx);
cudaStream_t context_stream(const p2z_context *ctx);
p2z_status context_fail(p2z_context *ctx, p2z_status st, const char *msg);
void *context_scratch(p2z_context *ctx, size_t bytes);
}  // namespace p2z

namespace {

constexpr int kLag = 31;
constexpr int kAttempts = 31 * 64;    // attempts per chunk (a whole number of 31-draw ring blocks per 2 blocks)
constexpr int kDraws = 2 * kAttempts;  // draws per chunk
constexpr int kThreads = 128;

// The 31 words a chunk starts from: slot j holds r[k0 - 31 + j], k0 = the
// chunk's first draw.  In that relative form the recurrence is
// r[k0 + i] = slot[i mod 31](old) + slot[(i + 28) mod 31] and the ring can be
// unrolled with compile-time slot numbers.
struct State {
  uint32_t w[kLag];
};

struct Seeds {
  float par[6];
  float cov[21];
  int32_t q;
  float hpos[32][3];
  float hcov[32][6];
};

struct Geometry {
  int B;
  int nlayer;
  int64_t nb;           // batches per event
  int64_t ntracks;      // nevts * ntrks
  int64_t nvar_trk;     // ntracks * 27
  int64_t nvar;         // + nlayer * ntracks * 9
  double smear, cov_scale;
};

// The chunk's attempts, two ring blocks (62 draws, 31 attempts) at a time:
// f(attempt index within the chunk, draw 1, draw 2).
template <class F>
__device__ __forceinline__ void for_each_attempt(State st, F f) {
  uint32_t s[kLag];
#pragma unroll
  for (int i = 0; i < kLag; ++i) s[i] = st.w[i];
  for (int blk = 0; blk < kAttempts / kLag; ++blk) {
    uint32_t d, prev = 0;
    int a = blk * kLag;
#pragma unroll
    for (int i = 0; i < 2 * kLag; ++i) {
      const int slot = i % kLag;
      s[slot] += s[(slot + 28) % kLag];
      d = s[slot] >> 1;
      if (i & 1) f(a++, (int32_t)prev, (int32_t)d);
      else prev = d;
    }
  }
}

__device__ __forceinline__ bool accepted(int32_t d1, int32_t d2, float *u1, float *u2, float *w) {
  *w = p2z_refrng::attempt(d1, d2, u1, u2);
  return !(*w >= 1 || *w == 0);
}

__global__ void __launch_bounds__(kThreads) k_count(const State *states, int nchunks, uint32_t *counts) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nchunks) return;
  uint32_t n = 0;
  for_each_attempt(states[c], [&](int, int32_t d1, int32_t d2) {
    float u1, u2, w;
    n += accepted(d1, d2, &u1, &u2, &w) ? 1u : 0u;
  });
  counts[c] = n;
}

// Variate v's output word: its address and the seed element it smears.
__device__ __forceinline__ void write_variate(const Geometry &g, const Seeds &sd, float *trk, float *hits, int64_t v,
                                              float r) {
  const double sf = fma(g.smear, (double)r, 1.0);  // the reference's (1 + smear*randn), one rounding
  const int B = g.B;
  if (v < g.nvar_trk) {
    const int64_t t = v / 27;
    const int ip = (int)(v - t * 27);
    const int64_t batch = t / B;  // batches of an event are consecutive: ib + nb*ie
    const int it = (int)(t - batch * B);
    float *w = trk + batch * (int64_t)(28 * B) + (int64_t)ip * B + it;
    *w = ip < 6 ? (float)(sf * sd.par[ip]) : (float)(sf * sd.cov[ip - 6] * g.cov_scale);
  } else {
    const int64_t u = v - g.nvar_trk;
    const int64_t h = u / 9;
    const int ip = (int)(u - h * 9);
    const int lay = (int)(h / g.ntracks);
    const int64_t t = h - (int64_t)lay * g.ntracks;  // track index: event, batch, lane
    const int64_t batch = t / B;
    const int it = (int)(t - batch * B);
    float *w = hits + (lay + (int64_t)g.nlayer * batch) * (int64_t)(9 * B) + (int64_t)ip * B + it;
    *w = ip < 3 ? (float)(sf * sd.hpos[lay][ip]) : (float)(sf * sd.hcov[lay][ip - 3]);
  }
}

__global__ void __launch_bounds__(kThreads) k_emit(const State *states, const uint64_t *first, int nchunks,
                                                   Geometry g, const Seeds *seeds, float *trk, float *hits) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nchunks) return;
  const Seeds &sd = *seeds;
  uint64_t a = first[c];  // global index of this chunk's first accepted attempt
  for_each_attempt(states[c], [&](int, int32_t d1, int32_t d2) {
    float u1, u2, w;
    if (!accepted(d1, d2, &u1, &u2, &w)) return;
    const int64_t v = 2 * (int64_t)a++;
    if (v >= g.nvar) return;
    const float lg = (float)log((double)w);
    const float mult = sqrtf((-2 * lg) / w);
    write_variate(g, sd, trk, hits, v, 0.f + 1.f * (u1 * mult));
    if (v + 1 < g.nvar) write_variate(g, sd, trk, hits, v + 1, 0.f + 1.f * (u2 * mult));
  });
}

__global__ void k_charge(float *trk, int64_t ntracks, int B, int32_t q) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntracks) return;
  const int64_t batch = t / B;
  reinterpret_cast<int32_t *>(trk)[batch * 28 * B + 27 * B + (t - batch * B)] = q;
}

// 31x31 matrices over Z/2^32 acting on the relative state (new word = w[0] + w[28]).
using Mat = std::vector<uint32_t>;
Mat mat_mul(const Mat &a, const Mat &b) {
  Mat c(kLag * kLag, 0u);
  for (int i = 0; i < kLag; ++i)
    for (int k = 0; k < kLag; ++k) {
      const uint32_t aik = a[i * kLag + k];
      if (!aik) continue;
      for (int j = 0; j < kLag; ++j) c[i * kLag + j] += aik * b[k * kLag + j];
    }
  return c;
}

// M^draws, M the one-draw step: w'[j] = w[j+1] (j < 30), w'[30] = w[0] + w[28].
Mat step_power(int64_t draws) {
  Mat m(kLag * kLag, 0u), r(kLag * kLag, 0u);
  for (int j = 0; j + 1 < kLag; ++j) m[j * kLag + j + 1] = 1u;
  m[30 * kLag + 0] = 1u;
  m[30 * kLag + 28] += 1u;
  for (int i = 0; i < kLag; ++i) r[i * kLag + i] = 1u;
  for (; draws; draws >>= 1) {
    if (draws & 1) r = mat_mul(r, m);
    m = mat_mul(m, m);
  }
  return r;
}

State advance(const Mat &p, const State &s) {
  State o;
  for (int i = 0; i < kLag; ++i) {
    uint32_t acc = 0;
    for (int j = 0; j < kLag; ++j) acc += p[i * kLag + j] * s.w[j];
    o.w[i] = acc;
  }
  return o;
}

#define PP_CUDA(call)                                                            \
  do {                                                                           \
    cudaError_t e_ = (call);                                                     \
    if (e_ != cudaSuccess) {                                                     \
      char m_[256];                                                              \
      std::snprintf(m_, sizeof m_, "%s: %s", #call, cudaGetErrorString(e_));     \
      return p2z::context_fail(ctx, P2Z_CUDA_ERROR, m_);                         \
    }                                                                            \
  } while (0)

}  // namespace

extern "C" p2z_status p2z_prepare_device(p2z_context *ctx, const p2z_atrk *seed, const p2z_ahit *hit_seeds,
                                         int nseeds, int bsize, int64_t nevts, int64_t ntrks, int nlayer,
                                         double smear, double cov_scale, void *d_trk_out, void *d_hits_out,
                                         void *stream) {
  if (!ctx) return P2Z_BAD_ARG;
  if (!seed || !hit_seeds) return p2z::context_fail(ctx, P2Z_BAD_ARG, "NULL seed");
  if (!(bsize == 8 || bsize == 16 || bsize == 32 || bsize == 64))
    return p2z::context_fail(ctx, P2Z_UNSUPPORTED, "bsize not in {8,16,32,64}");
  if (nevts < 0 || ntrks < 0 || ntrks % bsize || nlayer < 1 || nlayer > 32)
    return p2z::context_fail(ctx, P2Z_BAD_ARG, "bad sizes");
  if (nseeds < nlayer) return p2z::context_fail(ctx, P2Z_BAD_ARG, "fewer hit seeds than layers");
  Geometry g;
  g.B = bsize;
  g.nlayer = nlayer;
  g.nb = ntrks / bsize;
  g.ntracks = nevts * ntrks;
  g.nvar_trk = g.ntracks * 27;
  g.nvar = g.nvar_trk + (int64_t)nlayer * g.ntracks * 9;
  g.smear = smear;
  g.cov_scale = cov_scale;
  if (g.ntracks == 0) return P2Z_OK;
  if (!d_trk_out || !d_hits_out) return p2z::context_fail(ctx, P2Z_BAD_ARG, "NULL device buffer");
  PP_CUDA(cudaSetDevice(p2z::context_device(ctx)));
  cudaStream_t st = stream ? (cudaStream_t)stream : p2z::context_stream(ctx);

  Seeds sd;
  std::memcpy(sd.par, seed->par, sizeof sd.par);
  std::memcpy(sd.cov, seed->cov, sizeof sd.cov);
  sd.q = seed->q;
  for (int l = 0; l < nlayer; ++l) {
    std::memcpy(sd.hpos[l], hit_seeds[l].pos, sizeof sd.hpos[l]);
    std::memcpy(sd.hcov[l], hit_seeds[l].cov, sizeof sd.hcov[l]);
  }
  // Accepted attempts needed: nvar/2 rounded up; attempts are accepted with
  // probability pi/4.  Chunks for that many attempts plus 6 standard
  // deviations; more are added if the count falls short.
  const double need = (double)((g.nvar + 1) / 2);
  const double att = need / 0.7853981633974483;
  int64_t nchunks = (int64_t)std::ceil((att + 6.0 * std::sqrt(att) + 1.0) / kAttempts);
  const Mat jump = step_power(kDraws);
  std::vector<State> states;
  {
    p2z_ref_rng r;
    p2z_refrng::seed(&r, 1u);  // srand(1): the reference's initial state
    State s0;
    for (int j = 0; j < kLag; ++j) s0.w[j] = r.ring[(r.next - kLag + j) % kLag];
    states.push_back(s0);
  }
  for (int pass = 0; pass < 4; ++pass) {
    while ((int64_t)states.size() < nchunks) states.push_back(advance(jump, states.back()));
    // scratch: states, then the per-chunk counts / first indices (uint64), then
    // the seeds, each part starting on a 256-byte boundary (sizeof(State) is
    // 124, so the parts' sizes are rounded up)
    auto up256 = [](size_t n) { return (n + 255) / 256 * 256; };
    const size_t sbytes = up256(sizeof(State) * (size_t)nchunks), cbytes = up256(sizeof(uint64_t) * (size_t)nchunks);
    char *scr = static_cast<char *>(p2z::context_scratch(ctx, sbytes + cbytes + up256(sizeof(Seeds))));
    if (!scr) return P2Z_OOM;
    State *d_states = reinterpret_cast<State *>(scr);
    uint64_t *d_first = reinterpret_cast<uint64_t *>(scr + sbytes);
    Seeds *d_seeds = reinterpret_cast<Seeds *>(scr + sbytes + cbytes);
    PP_CUDA(cudaMemcpyAsync(d_states, states.data(), sizeof(State) * (size_t)nchunks, cudaMemcpyHostToDevice, st));
    const unsigned grid = (unsigned)((nchunks + kThreads - 1) / kThreads);
    uint32_t *d_counts = reinterpret_cast<uint32_t *>(d_first);  // counts, then the prefix sum in place
    k_count<<<grid, kThreads, 0, st>>>(d_states, (int)nchunks, d_counts);
    PP_CUDA(cudaGetLastError());
    std::vector<uint32_t> counts((size_t)nchunks);
    PP_CUDA(cudaMemcpyAsync(counts.data(), d_counts, sizeof(uint32_t) * (size_t)nchunks, cudaMemcpyDeviceToHost, st));
    PP_CUDA(cudaStreamSynchronize(st));
    std::vector<uint64_t> first((size_t)nchunks);
    uint64_t acc = 0;
    for (int64_t c = 0; c < nchunks; ++c) {
      first[(size_t)c] = acc;
      acc += counts[(size_t)c];
    }
    if ((double)acc < need) {  // rare: draw more chunks and count again
      nchunks += nchunks / 16 + 1;
      continue;
    }
    PP_CUDA(cudaMemcpyAsync(d_first, first.data(), sizeof(uint64_t) * (size_t)nchunks, cudaMemcpyHostToDevice, st));
    PP_CUDA(cudaMemcpyAsync(d_seeds, &sd, sizeof sd, cudaMemcpyHostToDevice, st));
    k_emit<<<grid, kThreads, 0, st>>>(d_states, d_first, (int)nchunks, g, d_seeds, (float *)d_trk_out,
                                      (float *)d_hits_out);
    PP_CUDA(cudaGetLastError());
    k_charge<<<(unsigned)((g.ntracks + 255) / 256), 256, 0, st>>>((float *)d_trk_out, g.ntracks, bsize, sd.q);
    PP_CUDA(cudaGetLastError());
    PP_CUDA(cudaStreamSynchronize(st));
    return P2Z_OK;
  }
  return p2z::context_fail(ctx, P2Z_CUDA_ERROR, "the random stream fell short of the variates needed");
}
