/*
 * p2z_types.hpp -- the reference benchmark's typed surface (C++17, header
 * only) over the C ABI of p2z.h, so that the reference's own host code can call
 * the B200 library with its own names.
 *
 * The reference fixes bsize, nevts, ntrks and nlayer as macros and defines its
 * matriplex structs per translation unit (src/propagate-toz-test_OMP.cpp:
 * 69-125).  Here the batch width is a template parameter B (8, 16, 32 or 64)
 * and the event sizes are run-time values carried by the owning arrays:
 *
 *   reference                                  here
 *   ---------------------------------------    -------------------------------------------
 *   struct MP6F, MP6x6SF, MP1I, MP3F, ...      p2z::MP6F<B>, p2z::MP6x6SF<B>, ...   (same bytes)
 *   struct MPTRK { par; cov; q; }  (:113-118)  p2z::MPTRK<B>                        (same bytes)
 *   struct MPHIT { pos; cov; }     (:120-123)  p2z::MPHIT<B>                        (same bytes)
 *   struct ALLTRKS / ALLHITS (backup/propagate-toz-test.h:79-91)
 *                                              p2z::ALLTRKS<B> / p2z::ALLHITS<B>: owning
 *                                              arrays of nevts*nb MPTRK / nlayer*nevts*nb MPHIT
 *   bTk(tracks, ev, ib), bHit(hits, ev, ib, lay) (:147-153, :212-217)
 *                                              ALLTRKS::bTk, ALLHITS::bHit
 *   srand(1); prepareTracks(ATRK) (:243)       p2z::RefRandom rng(1); prepareTracks<B>(trk, nevts, ntrks, rng)
 *   prepareHits(std::vector<AHIT>&) (:265)     prepareHits<B>(hits, nevts, ntrks, nlayer, rng)
 *   propagateToZ(&cov, &par, &q, &msP, &cov, &par) (:623), on one batch
 *                                              propagateToZ(DeviceTracks&, const DeviceHits&, layer):
 *                                              every batch of the array, on the GPU
 *   KalmanUpdate_v2(&cov, &par, &hitcov, &msP) (:503)
 *                                              KalmanUpdate_v2(DeviceTracks&, const DeviceHits&, layer)
 *   the timed loop over events, batches, layers (:731-748)
 *                                              p2z::run(device, trk, hit, out[, options])
 *   the printed validation block (:758-876)    p2z::validate(out, hit_last), p2z::print_validation
 *
 * propagateToZ / KalmanUpdate_v2 here evaluate the reference's own FP32
 * expressions with every operation separately rounded (p2z_step_device):
 * layer-by-layer driving reproduces the reference built without FMA
 * contraction.  p2z::run takes the fused path (all layers in one pass, the
 * precise evaluation unless options ask for the reference's rounding).
 * Errors are thrown as p2z::Error with the library's status and message.
 */
#ifndef P2Z_TYPES_HPP
#define P2Z_TYPES_HPP

/* The reference's sources define their sizes as macros (bsize, nevts, ntrks,
 * nlayer, nb, NITER, nthreads, smear, N: src/propagate-toz-test_OMP.cpp:18-41,
 * :296) before any code; they are set aside here, so this header can be
 * included after them, and restored at its end. */
#pragma push_macro("bsize")
#undef bsize
#pragma push_macro("nevts")
#undef nevts
#pragma push_macro("ntrks")
#undef ntrks
#pragma push_macro("nlayer")
#undef nlayer
#pragma push_macro("nb")
#undef nb
#pragma push_macro("NITER")
#undef NITER
#pragma push_macro("nthreads")
#undef nthreads
#pragma push_macro("smear")
#undef smear
#pragma push_macro("N")
#undef N

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "p2z.h"

namespace p2z {

/* ---- errors ------------------------------------------------------------- */

class Error : public std::runtime_error {
 public:
  Error(p2z_status s, const std::string &msg)
      : std::runtime_error(std::string(p2z_status_string(s)) + (msg.empty() ? "" : ": " + msg)), status(s) {}
  p2z_status status;
};

inline void check(p2z_status s, const p2z_context *ctx = nullptr) {
  if (s != P2Z_OK) throw Error(s, p2z_last_error(ctx));
}

/* ---- the matriplex types (element e of lane t at data[t + e*B]) ---------- */

template <int B> struct MP1I { int32_t data[1 * B]; };
template <int B> struct MP22I { int32_t data[22 * B]; };
template <int B> struct MP2F { float data[2 * B]; };
template <int B> struct MP3F { float data[3 * B]; };
template <int B> struct MP6F { float data[6 * B]; };
template <int B> struct MP2x2SF { float data[3 * B]; };
template <int B> struct MP2x6 { float data[12 * B]; };
template <int B> struct MP3x3 { float data[9 * B]; };
template <int B> struct MP3x3SF { float data[6 * B]; };
template <int B> struct MP3x6 { float data[18 * B]; };
template <int B> struct MP6x6SF { float data[21 * B]; };
template <int B> struct MP6x6F { float data[36 * B]; };

template <int B> struct MPTRK {
  MP6F<B> par;
  MP6x6SF<B> cov;
  MP1I<B> q;
};

template <int B> struct MPHIT {
  MP3F<B> pos;
  MP3x3SF<B> cov;
};

using ATRK = p2z_atrk;
using AHIT = p2z_ahit;

template <int B> constexpr bool valid_bsize() { return B == 8 || B == 16 || B == 32 || B == 64; }

#define P2Z_TYPES_CHECK(B)                                                                             \
  static_assert(sizeof(MPTRK<B>) == 28 * (B) * 4, "MPTRK layout");                                  \
  static_assert(sizeof(MPHIT<B>) == 9 * (B) * 4, "MPHIT layout");                                   \
  static_assert(offsetof(MPTRK<B>, cov) == 6 * (B) * 4 && offsetof(MPTRK<B>, q) == 27 * (B) * 4,    \
                "MPTRK field offsets");                                                             \
  static_assert(offsetof(MPHIT<B>, cov) == 3 * (B) * 4, "MPHIT field offsets");
P2Z_TYPES_CHECK(8)
P2Z_TYPES_CHECK(16)
P2Z_TYPES_CHECK(32)
P2Z_TYPES_CHECK(64)
#undef P2Z_TYPES_CHECK
static_assert(sizeof(ATRK) == 112 && sizeof(AHIT) == 36, "ATRK / AHIT layout");

/* Packed lower-triangle index of (i, j) in a symmetric 6x6 (SymOffsets66, :52-55). */
constexpr int sym66(int i, int j) { return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; }

/* ---- element accessors (:155-231) ------------------------------------------ */

template <int B> inline float par(const MPTRK<B> *b, size_t it, size_t ip) { return b->par.data[it + ip * B]; }
template <int B> inline float x(const MPTRK<B> *b, size_t it) { return par(b, it, 0); }
template <int B> inline float y(const MPTRK<B> *b, size_t it) { return par(b, it, 1); }
template <int B> inline float z(const MPTRK<B> *b, size_t it) { return par(b, it, 2); }
template <int B> inline float ipt(const MPTRK<B> *b, size_t it) { return par(b, it, 3); }
template <int B> inline float phi(const MPTRK<B> *b, size_t it) { return par(b, it, 4); }
template <int B> inline float theta(const MPTRK<B> *b, size_t it) { return par(b, it, 5); }
template <int B> inline int q(const MPTRK<B> *b, size_t it) { return b->q.data[it]; }
template <int B> inline float cov(const MPTRK<B> *b, size_t it, int i, int j) {
  return b->cov.data[it + sym66(i, j) * B];
}
template <int B> inline float pos(const MPHIT<B> *h, size_t it, size_t ip) { return h->pos.data[it + ip * B]; }
template <int B> inline void setpar(MPTRK<B> *b, size_t it, size_t ip, float v) { b->par.data[it + ip * B] = v; }

/* ---- page-locked host memory ------------------------------------------------ */

namespace detail {
struct HostBuffer {
  void *p = nullptr;
  size_t bytes = 0;
  HostBuffer() = default;
  explicit HostBuffer(size_t n) : bytes(n) { check(p2z_host_alloc(&p, n)); }
  HostBuffer(HostBuffer &&o) noexcept : p(std::exchange(o.p, nullptr)), bytes(std::exchange(o.bytes, 0)) {}
  HostBuffer &operator=(HostBuffer &&o) noexcept {
    if (this != &o) {
      p2z_host_free(p);
      p = std::exchange(o.p, nullptr);
      bytes = std::exchange(o.bytes, 0);
    }
    return *this;
  }
  HostBuffer(const HostBuffer &) = delete;
  HostBuffer &operator=(const HostBuffer &) = delete;
  ~HostBuffer() { p2z_host_free(p); }
};
}  // namespace detail

/* ---- ALLTRKS / ALLHITS: the event arrays ------------------------------------ */

/* nevts*nb track batches (nb = ntrks/B), batch ib of event ev at btrks[ib + nb*ev],
 * in page-locked host memory. */
template <int B> class ALLTRKS {
  static_assert(valid_bsize<B>(), "bsize must be 8, 16, 32 or 64");

 public:
  ALLTRKS() = default;
  ALLTRKS(int64_t nevts, int64_t ntrks)
      : buf_(sizeof(MPTRK<B>) * (size_t)(nevts * (ntrks / B))), nevts_(nevts), ntrks_(ntrks) {
    if (nevts < 0 || ntrks < 0 || ntrks % B) throw Error(P2Z_BAD_ARG, "ntrks must be a multiple of bsize");
    btrks = static_cast<MPTRK<B> *>(buf_.p);
  }
  MPTRK<B> *btrks = nullptr;
  MPTRK<B> *bTk(size_t ev, size_t ib) { return &btrks[ib + nb() * ev]; }
  const MPTRK<B> *bTk(size_t ev, size_t ib) const { return &btrks[ib + nb() * ev]; }
  int64_t nevts() const { return nevts_; }
  int64_t ntrks() const { return ntrks_; }
  int64_t nb() const { return ntrks_ / B; }
  int64_t nbatches() const { return nevts_ * nb(); }
  size_t bytes() const { return sizeof(MPTRK<B>) * (size_t)nbatches(); }
  /* element ip of track tk of event ev (reference :178-183) */
  float par(size_t ev, size_t tk, size_t ip) const { return p2z::par(bTk(ev, tk / B), tk % B, ip); }

 private:
  detail::HostBuffer buf_;
  int64_t nevts_ = 0, ntrks_ = 0;
};

/* nlayer*nevts*nb hit batches; the hits of batch ib of event ev on layer lay at
 * bhits[lay + nlayer*(ib + nb*ev)] (the layers of a batch are contiguous). */
template <int B> class ALLHITS {
  static_assert(valid_bsize<B>(), "bsize must be 8, 16, 32 or 64");

 public:
  ALLHITS() = default;
  ALLHITS(int64_t nevts, int64_t ntrks, int nlayer)
      : buf_(sizeof(MPHIT<B>) * (size_t)(nevts * (ntrks / B) * nlayer)),
        nevts_(nevts),
        ntrks_(ntrks),
        nlayer_(nlayer) {
    if (nevts < 0 || ntrks < 0 || ntrks % B || nlayer < 1 || nlayer > 32)
      throw Error(P2Z_BAD_ARG, "bad ALLHITS sizes");
    bhits = static_cast<MPHIT<B> *>(buf_.p);
  }
  MPHIT<B> *bhits = nullptr;
  const MPHIT<B> *bHit(size_t ev, size_t ib, size_t lay) const { return &bhits[lay + nlayer_ * (ib + nb() * ev)]; }
  MPHIT<B> *bHit(size_t ev, size_t ib, size_t lay) { return &bhits[lay + nlayer_ * (ib + nb() * ev)]; }
  int64_t nevts() const { return nevts_; }
  int64_t ntrks() const { return ntrks_; }
  int nlayer() const { return nlayer_; }
  int64_t nb() const { return ntrks_ / B; }
  int64_t nbatches() const { return nevts_ * nb(); }
  size_t bytes() const { return sizeof(MPHIT<B>) * (size_t)nbatches() * nlayer_; }

 private:
  detail::HostBuffer buf_;
  int64_t nevts_ = 0, ntrks_ = 0;
  int nlayer_ = 0;
};

/* ---- input preparation (:127-145, :243-293) --------------------------------- */

/* The reference's rand() / randn stream: RefRandom rng(1) is the state after
 * srand(1) (the C library's initial state), which the reference's main uses. */
class RefRandom {
 public:
  explicit RefRandom(uint32_t seed = 1) { p2z_ref_rng_seed(&g_, seed); }
  int32_t rand() { return p2z_ref_rng_rand(&g_); }
  float randn() { return p2z_ref_rng_randn(&g_); }
  p2z_ref_rng *get() { return &g_; }

 private:
  p2z_ref_rng g_;
};

/* prepareTracks (:243-263): every element times (1 + smear*randn), the
 * covariance also times cov_scale (the reference: 100); the charge copied. */
template <int B>
ALLTRKS<B> prepareTracks(const ATRK &inputtrk, int64_t nevts, int64_t ntrks, RefRandom &rng, double smear = 1e-7,
                         double cov_scale = 100.0) {
  ALLTRKS<B> t(nevts, ntrks);
  check(p2z_prepare_tracks(rng.get(), &inputtrk, B, nevts, ntrks, smear, cov_scale, t.btrks));
  return t;
}

/* prepareHits (:265-293): layer l from inputhits[l]; fewer hits than layers
 * is an Error (the reference exits). */
template <int B>
ALLHITS<B> prepareHits(const std::vector<AHIT> &inputhits, int64_t nevts, int64_t ntrks, int nlayer, RefRandom &rng,
                       double smear = 1e-7) {
  ALLHITS<B> h(nevts, ntrks, nlayer);
  check(p2z_prepare_hits(rng.get(), inputhits.data(), (int)inputhits.size(), B, nevts, ntrks, nlayer, smear,
                         h.bhits));
  return h;
}

/* ---- the device -------------------------------------------------------------- */

class Device {
 public:
  explicit Device(int device = -1) { check(p2z_create(device, &ctx_)); }
  Device(const Device &) = delete;
  Device &operator=(const Device &) = delete;
  ~Device() { p2z_destroy(ctx_); }
  p2z_context *get() const { return ctx_; }

 private:
  p2z_context *ctx_ = nullptr;
};

namespace detail {
struct DeviceBuffer {
  p2z_context *ctx = nullptr;
  void *p = nullptr;
  size_t bytes = 0;
  DeviceBuffer(p2z_context *c, size_t n) : ctx(c), bytes(n) { check(p2z_device_alloc(c, &p, n), c); }
  DeviceBuffer(DeviceBuffer &&o) noexcept
      : ctx(o.ctx), p(std::exchange(o.p, nullptr)), bytes(std::exchange(o.bytes, 0)) {}
  DeviceBuffer(const DeviceBuffer &) = delete;
  DeviceBuffer &operator=(const DeviceBuffer &) = delete;
  ~DeviceBuffer() {
    if (p) p2z_device_free(ctx, p);
  }
};
}  // namespace detail

/* Device copies of the event arrays, for driving the layer loop on the GPU. */
template <int B> class DeviceTracks {
 public:
  DeviceTracks(const Device &dev, const ALLTRKS<B> &host)
      : buf_(dev.get(), host.bytes()), nevts_(host.nevts()), ntrks_(host.ntrks()) {
    check(p2z_copy(dev.get(), buf_.p, host.btrks, host.bytes()), dev.get());
  }
  /* the current tracks, copied back to the host */
  ALLTRKS<B> download() const {
    ALLTRKS<B> out(nevts_, ntrks_);
    check(p2z_copy(buf_.ctx, out.btrks, buf_.p, out.bytes()), buf_.ctx);
    return out;
  }
  MPTRK<B> *btrks() { return static_cast<MPTRK<B> *>(buf_.p); }
  int64_t nbatches() const { return nevts_ * (ntrks_ / B); }
  p2z_context *ctx() const { return buf_.ctx; }

 private:
  detail::DeviceBuffer buf_;
  int64_t nevts_, ntrks_;
};

template <int B> class DeviceHits {
 public:
  DeviceHits(const Device &dev, const ALLHITS<B> &host) : buf_(dev.get(), host.bytes()), nlayer_(host.nlayer()) {
    check(p2z_copy(dev.get(), buf_.p, host.bhits, host.bytes()), dev.get());
  }
  const MPHIT<B> *bhits() const { return static_cast<const MPHIT<B> *>(buf_.p); }
  int nlayer() const { return nlayer_; }

 private:
  detail::DeviceBuffer buf_;
  int nlayer_;
};

/* propagateToZ (:623-682) of every track to its hit plane on `layer`, in
 * place, with the reference's field constant unless kfact is given. */
template <int B>
void propagateToZ(DeviceTracks<B> &trk, const DeviceHits<B> &hits, int layer, float kfact = 0.f) {
  check(p2z_step_device(trk.ctx(), B, trk.nbatches(), trk.btrks(), hits.bhits(), hits.nlayer(), layer, 1,
                        P2Z_UPDATE_V2, kfact),
        trk.ctx());
}

/* KalmanUpdate_v2 (:503-620) of every track with its hit on `layer`, in place. */
template <int B> void KalmanUpdate_v2(DeviceTracks<B> &trk, const DeviceHits<B> &hits, int layer) {
  check(p2z_step_device(trk.ctx(), B, trk.nbatches(), trk.btrks(), hits.bhits(), hits.nlayer(), layer, 2,
                        P2Z_UPDATE_V2, 0.f),
        trk.ctx());
}

/* ---- the whole pass --------------------------------------------------------- */

struct RunOptions {
  int niter = 1;
  p2z_update_kind update = P2Z_UPDATE_V2;
  uint32_t flags = 0;  /* P2Z_FLAG_*, e.g. P2Z_FLAG_REFERENCE_ROUNDING */
  float kfact = 0.f;
  /* launch shape; 0 / AUTO: what p2z_autotune measured best on the device, else the defaults */
  p2z_schedule schedule = P2Z_SCHED_AUTO;
  int block_threads = 0;
  int threads_per_track = 0;
};

/* The reference's timed loop (:731-748) -- for every event, batch and layer,
 * propagateToZ then the update -- from host arrays through p2z_run. */
template <int B>
p2z_stats run(const Device &dev, const ALLTRKS<B> &trk, const ALLHITS<B> &hit, ALLTRKS<B> &out,
              const RunOptions &o = RunOptions()) {
  if (trk.nevts() != hit.nevts() || trk.ntrks() != hit.ntrks() || out.nbatches() != trk.nbatches())
    throw Error(P2Z_BAD_ARG, "track, hit and output arrays describe different events");
  p2z_config c{};
  c.abi_version = P2Z_ABI_VERSION;
  c.bsize = B;
  c.nevts = trk.nevts();
  c.ntrks = trk.ntrks();
  c.nlayer = hit.nlayer();
  c.niter = o.niter;
  c.kfact = o.kfact;
  c.update = o.update;
  c.flags = o.flags;
  c.schedule = o.schedule;
  c.block_threads = o.block_threads;
  c.threads_per_track = o.threads_per_track;
  p2z_stats st{};
  check(p2z_run(dev.get(), &c, trk.btrks, hit.bhits, nullptr, out.btrks, &st), dev.get());
  return st;
}

/* ---- validation block (:758-876) -------------------------------------------- */

template <int B> p2z_validation validate(const ALLTRKS<B> &out, const AHIT &last_hit) {
  p2z_validation v{};
  check(p2z_validate(out.btrks, B, out.nevts(), out.ntrks(), last_hit.pos, &v));
  return v;
}

inline void print_validation(const p2z_validation &v) { p2z_print_validation(&v); }

}  // namespace p2z

#pragma pop_macro("bsize")
#pragma pop_macro("nevts")
#pragma pop_macro("ntrks")
#pragma pop_macro("nlayer")
#pragma pop_macro("nb")
#pragma pop_macro("NITER")
#pragma pop_macro("nthreads")
#pragma pop_macro("smear")
#pragma pop_macro("N")

#endif /* P2Z_TYPES_HPP */
