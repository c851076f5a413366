// p2z_host.cpp -- host-side pieces of the library: the reference-compatible
// input preparation (prepareTracks / prepareHits), the physics workload
// generator, layer masks for uneven workloads, and the validation block.
// None of this is on the device hot path; it builds inputs and checks outputs
// exactly as the reference's setup and reporting code does.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "p2z.h"
#include "p2z_gen.h"
#include "p2z_refrng.h"

namespace {

constexpr int TRK_WORDS = 28;
constexpr int HIT_WORDS = 9;

bool valid_bsize(int b) { return b == 8 || b == 16 || b == 32 || b == 64; }

// The reference's smearing factor (1 + smear*randn), formed in double.  Its
// builds compile with FMA contraction on (gcc -O3 -march=native), which turns
// this expression into one fused multiply-add; that rounding is kept here.
inline double smear_factor(double smear, float r) { return std::fma(smear, (double)r, 1.0); }

int host_threads(int requested) {
  if (requested > 0) return requested;
  const unsigned h = std::thread::hardware_concurrency();
  return h ? (int)h : 1;
}

template <class F>
void parallel_for(int64_t n, int nthr, F f) {
  nthr = (int)std::max<int64_t>(1, std::min<int64_t>(nthr, n));
  if (nthr <= 1) {
    f(0, n);
    return;
  }
  std::vector<std::thread> th;
  const int64_t chunk = (n + nthr - 1) / nthr;
  for (int t = 0; t < nthr; ++t) {
    const int64_t a = t * chunk, b = std::min(n, a + chunk);
    if (a >= b) break;
    th.emplace_back([=] { f(a, b); });
  }
  for (auto &x : th) x.join();
}

}  // namespace

extern "C" {

void p2z_ref_rng_seed(p2z_ref_rng *g, uint32_t seed) {
  if (g) p2z_refrng::seed(g, seed);
}

int32_t p2z_ref_rng_rand(p2z_ref_rng *g) { return g ? p2z_refrng::draw(g) : -1; }

float p2z_ref_rng_randn(p2z_ref_rng *g) { return g ? p2z_refrng::randn(g) : NAN; }

p2z_status p2z_prepare_tracks(p2z_ref_rng *g, const p2z_atrk *seed, int bsize, int64_t nevts, int64_t ntrks,
                              double smear, double cov_scale, void *trk_out) {
  if (!g || !seed || (!trk_out && nevts * ntrks > 0)) return P2Z_BAD_ARG;
  if (!valid_bsize(bsize)) return P2Z_UNSUPPORTED;
  if (nevts < 0 || ntrks < 0 || ntrks % bsize) return P2Z_BAD_ARG;
  const int64_t nb = ntrks / bsize;
  float *T = (float *)trk_out;
  // prepareTracks (src/propagate-toz-test_OMP.cpp:243-263): event, batch,
  // lane; 6 parameters then 21 covariance elements, each scaled by
  // (1 + smear*randn); covariance also by cov_scale (100 in the reference);
  // the charge copied.
  for (int64_t ie = 0; ie < nevts; ++ie)
    for (int64_t ib = 0; ib < nb; ++ib) {
      float *b = T + (ib + nb * ie) * (int64_t)TRK_WORDS * bsize;
      for (int it = 0; it < bsize; ++it) {
        for (int ip = 0; ip < 6; ++ip) b[it + ip * bsize] = smear_factor(smear, p2z_refrng::randn(g)) * seed->par[ip];
        for (int ip = 0; ip < 21; ++ip)
          b[6 * bsize + it + ip * bsize] = smear_factor(smear, p2z_refrng::randn(g)) * seed->cov[ip] * cov_scale;
        std::memcpy(&b[27 * bsize + it], &seed->q, sizeof(int32_t));
      }
    }
  return P2Z_OK;
}

p2z_status p2z_prepare_hits(p2z_ref_rng *g, const p2z_ahit *hit_seeds, int nseeds, int bsize, int64_t nevts,
                            int64_t ntrks, int nlayer, double smear, void *hits_out) {
  if (!g || !hit_seeds || (!hits_out && nevts * ntrks > 0)) return P2Z_BAD_ARG;
  if (!valid_bsize(bsize)) return P2Z_UNSUPPORTED;
  if (nevts < 0 || ntrks < 0 || ntrks % bsize || nlayer < 1 || nlayer > 32) return P2Z_BAD_ARG;
  if (nseeds < nlayer) return P2Z_BAD_ARG;  // the reference exits here (:271-274)
  const int64_t nb = ntrks / bsize;
  float *H = (float *)hits_out;
  // prepareHits (:265-293): layer outermost; layer l of batch ib of event ie
  // at hit batch l + nlayer*(ib + nb*ie).
  for (int lay = 0; lay < nlayer; ++lay) {
    const p2z_ahit &s = hit_seeds[lay];
    for (int64_t ie = 0; ie < nevts; ++ie)
      for (int64_t ib = 0; ib < nb; ++ib) {
        float *h = H + (lay + nlayer * (ib + nb * ie)) * (int64_t)HIT_WORDS * bsize;
        for (int it = 0; it < bsize; ++it) {
          for (int ip = 0; ip < 3; ++ip) h[it + ip * bsize] = smear_factor(smear, p2z_refrng::randn(g)) * s.pos[ip];
          for (int ip = 0; ip < 6; ++ip)
            h[3 * bsize + it + ip * bsize] = smear_factor(smear, p2z_refrng::randn(g)) * s.cov[ip];
        }
      }
  }
  return P2Z_OK;
}

p2z_status p2z_prepare(const p2z_atrk *seed, const p2z_ahit *hit_seeds, int nseeds, int bsize, int64_t nevts,
                       int64_t ntrks, int nlayer, double smear, double cov_scale, void *trk_out, void *hits_out) {
  if (!seed || !hit_seeds || !trk_out || !hits_out) return P2Z_BAD_ARG;
  if (!valid_bsize(bsize)) return P2Z_UNSUPPORTED;
  if (nevts < 0 || ntrks < 0 || ntrks % bsize || nlayer < 1 || nlayer > 32) return P2Z_BAD_ARG;
  if (nseeds < nlayer) return P2Z_BAD_ARG;
  // the reference's main: rand() in its initial state (srand(1)), then
  // prepareTracks, then prepareHits on the same stream (:715-720)
  p2z_ref_rng g;
  p2z_refrng::seed(&g, 1u);
  p2z_status r = p2z_prepare_tracks(&g, seed, bsize, nevts, ntrks, smear, cov_scale, trk_out);
  if (r != P2Z_OK) return r;
  return p2z_prepare_hits(&g, hit_seeds, nseeds, bsize, nevts, ntrks, nlayer, smear, hits_out);
}

void p2z_physics_defaults(p2z_physics_params *p) {
  if (!p) return;
  std::memset(p, 0, sizeof *p);
  p->seed = 20240601ull;
  p->pt_min = 0.5;
  p->pt_max = 20.0;
  p->eta_min = 1.6;
  p->eta_max = 2.5;
  p->sigma_vz = 5.0;
  p->sig_xy = 0.01;
  p->sig_z = 0.05;
  p->rel_sig_ipt = 0.01;
  p->sig_phi = 1e-3;
  p->sig_theta = 1e-3;
  p->rho_max = 0.3;
  p->z_first = 30.0;
  p->z_last = 270.0;
  p->hit_sig_xy = 30e-4;  // 30 um in cm
  p->hit_sig_z = 1e-4;    // 1 um in cm
  p->kfact = 0.f;
  p->nthreads = 0;
}

p2z_status p2z_generate_physics(const p2z_physics_params *p, const p2z_config *cfg, void *trk_out, void *hits_out,
                                uint32_t *hit_mask) {
  if (!p || !cfg || !trk_out || !hits_out) return P2Z_BAD_ARG;
  if (!valid_bsize(cfg->bsize)) return P2Z_UNSUPPORTED;
  const int B = cfg->bsize, nlayer = cfg->nlayer;
  if (nlayer < 1 || nlayer > 32 || cfg->nevts < 0) return P2Z_BAD_ARG;
  if (p->pt_min <= 0 || p->pt_max < p->pt_min || p->eta_max < p->eta_min) return P2Z_BAD_ARG;
  // event -> [first slot, number of real tracks)
  std::vector<int64_t> ev_first(cfg->nevts), ev_n(cfg->nevts);
  int64_t nb = 0;
  for (int64_t e = 0; e < cfg->nevts; ++e) {
    const int64_t n = cfg->event_ntrks ? cfg->event_ntrks[e] : cfg->ntrks;
    if (n < 0 || (!cfg->event_ntrks && n % B)) return P2Z_BAD_ARG;
    ev_first[e] = nb * B;
    ev_n[e] = n;
    nb += (n + B - 1) / B;
  }
  const int64_t nslots = nb * B;
  // slot -> event lookup through the batch's event
  std::vector<int64_t> batch_event(nb);
  for (int64_t e = 0; e < cfg->nevts; ++e) {
    const int64_t b0 = ev_first[e] / B, nbe = (ev_n[e] + B - 1) / B;
    for (int64_t i = 0; i < nbe; ++i) batch_event[b0 + i] = e;
  }
  const double kf = p->kfact != 0.f ? p->kfact : (double)(float)(100. / (-0.299792458 * 3.8112));
  const uint32_t all = nlayer >= 32 ? 0xffffffffu : ((1u << nlayer) - 1u);
  float *T = (float *)trk_out;
  float *H = (float *)hits_out;
  parallel_for(nslots, host_threads(p->nthreads), [&](int64_t s0, int64_t s1) {
    for (int64_t s = s0; s < s1; ++s) {
      const int64_t b = s / B;
      const int t = (int)(s % B);
      const p2z_gen::SlotView view{T + b * (int64_t)TRK_WORDS * B, H + b * nlayer * (int64_t)HIT_WORDS * B, t, B};
      const int64_t e = batch_event[b];
      const bool real = (s - ev_first[e]) < ev_n[e];
      if (!real) {
        p2z_gen::zero_slot(nlayer, view);
        if (hit_mask) hit_mask[s] = 0u;
        continue;
      }
      p2z_gen::generate_slot(*p, kf, nlayer, (uint64_t)s, view);
      if (hit_mask) hit_mask[s] = all;
    }
  });
  return P2Z_OK;
}

p2z_status p2z_mask_layers(uint32_t *hit_mask, int64_t nslots, int nlayer, int min_hits, int max_hits,
                           double drop_prob, uint64_t seed) {
  if (!hit_mask && nslots > 0) return P2Z_BAD_ARG;
  if (nlayer < 1 || nlayer > 32 || min_hits < 1 || max_hits < min_hits || max_hits > nlayer || drop_prob < 0 ||
      drop_prob >= 1)
    return P2Z_BAD_ARG;
  parallel_for(nslots, host_threads(0), [&](int64_t s0, int64_t s1) {
    for (int64_t s = s0; s < s1; ++s) {
      if (hit_mask[s] == 0u) continue;
      hit_mask[s] = p2z_gen::mask_slot(seed, (uint64_t)s, min_hits, max_hits, drop_prob);
    }
  });
  return P2Z_OK;
}

p2z_status p2z_validate_partial(const void *trk_out, int bsize, int64_t nevts, int64_t ntrks, const float hit_last[3],
                                const double means[6], p2z_validation_partial *acc) {
  if (!trk_out || !hit_last || !acc) return P2Z_BAD_ARG;
  if (!valid_bsize(bsize)) return P2Z_UNSUPPORTED;
  if (nevts < 0 || ntrks < 0 || ntrks % bsize) return P2Z_BAD_ARG;
  std::memset(acc, 0, sizeof *acc);
  const float *T = (const float *)trk_out;
  const int64_t nb = ntrks / bsize;
  const double hx_ = hit_last[0], hy_ = hit_last[1], hz_ = hit_last[2];
  // The reference's track selection (src/propagate-toz-test_OMP.cpp:758-864):
  // skip non-finite tracks, skip tracks outside its fixed window (pt ~ 12,
  // phi ~ 1.3, theta ~ 2.8, positions within 100% of the last seed hit).
  for (int64_t ie = 0; ie < nevts; ++ie)
    for (int64_t it = 0; it < ntrks; ++it) {
      const float *b = T + ((it / bsize) + nb * ie) * (int64_t)TRK_WORDS * bsize + (it % bsize);
      const double x_ = b[0], y_ = b[bsize], z_ = b[2 * bsize];
      const double pt_ = 1. / b[3 * bsize], phi_ = b[4 * bsize], theta_ = b[5 * bsize];
      if (!(std::isfinite(x_) && std::isfinite(y_) && std::isfinite(z_) && std::isfinite(pt_) &&
            std::isfinite(phi_) && std::isfinite(theta_))) {
        acc->nnans++;
        continue;
      }
      if (std::fabs((x_ - hx_) / hx_) > 1. || std::fabs((y_ - hy_) / hy_) > 1. || std::fabs((z_ - hz_) / hz_) > 1. ||
          std::fabs((pt_ - 12.) / 12.) > 1. || std::fabs((phi_ - 1.3) / 1.3) > 1. ||
          std::fabs((theta_ - 2.8) / 2.8) > 1.) {
        acc->nfail++;
        continue;
      }
      const double dx = (x_ - hx_) / x_, dy = (y_ - hy_) / y_, dz = (z_ - hz_) / z_;
      if (!means) {
        acc->sum[0] += x_;
        acc->sum[1] += y_;
        acc->sum[2] += z_;
        acc->sum[3] += dx;
        acc->sum[4] += dy;
        acc->sum[5] += dz;
        acc->sum[6] += pt_;
        acc->sum[7] += phi_;
        acc->sum[8] += theta_;
      } else {
        acc->sq[0] += (x_ - means[0]) * (x_ - means[0]);
        acc->sq[1] += (y_ - means[1]) * (y_ - means[1]);
        acc->sq[2] += (z_ - means[2]) * (z_ - means[2]);
        acc->sq[3] += (dx - means[3]) * (dx - means[3]);
        acc->sq[4] += (dy - means[4]) * (dy - means[4]);
        acc->sq[5] += (dz - means[5]) * (dz - means[5]);
      }
      acc->ngood++;
    }
  return P2Z_OK;
}

void p2z_validate_means(const p2z_validation_partial *p1, double means[6]) {
  for (int i = 0; i < 6; ++i) means[i] = p1->sum[i] / double(p1->ngood);
}

p2z_status p2z_validate_combine(const p2z_validation_partial *p1, const p2z_validation_partial *p2, p2z_validation *v) {
  if (!p1 || !p2 || !v) return P2Z_BAD_ARG;
  const double n = double(p1->ngood);
  v->avgx = p1->sum[0] / n;
  v->avgy = p1->sum[1] / n;
  v->avgz = p1->sum[2] / n;
  v->avgdx = p1->sum[3] / n;
  v->avgdy = p1->sum[4] / n;
  v->avgdz = p1->sum[5] / n;
  v->avgpt = p1->sum[6] / n;
  v->avgphi = p1->sum[7] / n;
  v->avgtheta = p1->sum[8] / n;
  // The reference takes these roots with sqrtf, i.e. in single precision.
  v->stdx = sqrtf((float)(p2->sq[0] / n));
  v->stdy = sqrtf((float)(p2->sq[1] / n));
  v->stdz = sqrtf((float)(p2->sq[2] / n));
  v->stddx = sqrtf((float)(p2->sq[3] / n));
  v->stddy = sqrtf((float)(p2->sq[4] / n));
  v->stddz = sqrtf((float)(p2->sq[5] / n));
  v->nnans = p1->nnans;
  v->nfail = p1->nfail;
  v->ngood = p1->ngood;
  return P2Z_OK;
}

p2z_status p2z_validate(const void *trk_out, int bsize, int64_t nevts, int64_t ntrks, const float hit_last[3],
                        p2z_validation *v) {
  if (!v) return P2Z_BAD_ARG;
  p2z_validation_partial p1, p2;
  p2z_status r = p2z_validate_partial(trk_out, bsize, nevts, ntrks, hit_last, nullptr, &p1);
  if (r != P2Z_OK) return r;
  double means[6];
  p2z_validate_means(&p1, means);
  r = p2z_validate_partial(trk_out, bsize, nevts, ntrks, hit_last, means, &p2);
  if (r != P2Z_OK) return r;
  return p2z_validate_combine(&p1, &p2, v);
}

void p2z_print_validation(const p2z_validation *v) {
  if (!v) return;
  // Text of the reference's block, line for line (:866-876).
  std::printf("track x avg=%f std/avg=%f\n", v->avgx, std::fabs(v->stdx / v->avgx));
  std::printf("track y avg=%f std/avg=%f\n", v->avgy, std::fabs(v->stdy / v->avgy));
  std::printf("track z avg=%f std/avg=%f\n", v->avgz, std::fabs(v->stdz / v->avgz));
  std::printf("track dx/x avg=%f std=%f\n", v->avgdx, v->stddx);
  std::printf("track dy/y avg=%f std=%f\n", v->avgdy, v->stddy);
  std::printf("track dz/z avg=%f std=%f\n", v->avgdz, v->stddz);
  std::printf("track pt avg=%f\n", v->avgpt);
  std::printf("track phi avg=%f\n", v->avgphi);
  std::printf("track theta avg=%f\n", v->avgtheta);
  std::printf("number of tracks with nans=%i\n", (int)v->nnans);
  std::printf("number of tracks failed=%i\n", (int)v->nfail);
  std::fflush(stdout);
}

p2z_status p2z_dump_tracks(const void *trk_in, const void *trk_out, int bsize, int64_t nevts, int64_t ntrks,
                           const float hit_last[3], const char *dir) {
  if (!trk_in || !trk_out || !hit_last) return P2Z_BAD_ARG;
  if (!valid_bsize(bsize)) return P2Z_UNSUPPORTED;
  if (nevts < 0 || ntrks < 0 || ntrks % bsize) return P2Z_BAD_ARG;
  const std::string base = (dir && *dir) ? std::string(dir) + "/" : std::string();
  static const char *names[6] = {"output_x.txt", "output_y.txt", "output_z.txt",
                                 "input_x.txt",  "input_y.txt",  "input_z.txt"};
  FILE *f[6] = {};
  for (int i = 0; i < 6; ++i) {
    f[i] = std::fopen((base + names[i]).c_str(), "w");
    if (!f[i]) {
      for (int j = 0; j < i; ++j) std::fclose(f[j]);
      return P2Z_BAD_ARG;
    }
  }
  const float *O = (const float *)trk_out, *I = (const float *)trk_in;
  const int64_t nb = ntrks / bsize;
  const double hx_ = hit_last[0], hy_ = hit_last[1], hz_ = hit_last[2];
  // the validation's selection (src/propagate-toz-test_OMP.cpp:758-795); the
  // dump's lines (src/propagate-toz-test_CUDA_v4.cu:1051-1055, :1129-1136)
  for (int64_t ie = 0; ie < nevts; ++ie)
    for (int64_t it = 0; it < ntrks; ++it) {
      const int64_t off = ((it / bsize) + nb * ie) * (int64_t)TRK_WORDS * bsize + (it % bsize);
      const float *b = O + off;
      const double x_ = b[0], y_ = b[bsize], z_ = b[2 * bsize];
      const double pt_ = 1. / b[3 * bsize], phi_ = b[4 * bsize], theta_ = b[5 * bsize];
      if (!(std::isfinite(x_) && std::isfinite(y_) && std::isfinite(z_) && std::isfinite(pt_) &&
            std::isfinite(phi_) && std::isfinite(theta_)))
        continue;
      if (std::fabs((x_ - hx_) / hx_) > 1. || std::fabs((y_ - hy_) / hy_) > 1. || std::fabs((z_ - hz_) / hz_) > 1. ||
          std::fabs((pt_ - 12.) / 12.) > 1. || std::fabs((phi_ - 1.3) / 1.3) > 1. ||
          std::fabs((theta_ - 2.8) / 2.8) > 1.)
        continue;
      const float *a = I + off;
      std::fprintf(f[0], "%f\n", x_);
      std::fprintf(f[1], "%f\n", y_);
      std::fprintf(f[2], "%f\n", z_);
      std::fprintf(f[3], "%f\n", (double)a[0]);
      std::fprintf(f[4], "%f\n", (double)a[bsize]);
      std::fprintf(f[5], "%f\n", (double)a[2 * bsize]);
    }
  for (int i = 0; i < 6; ++i) std::fclose(f[i]);
  return P2Z_OK;
}

void p2z_print_formatted(int niter, int64_t nevts, int64_t ntrks, int bsize, double wall_s, double setup_s,
                         int nthreads) {
  // The reference's machine-readable line (:756), read positionally by its
  // tools (tools/compare.py:12).
  std::printf("formatted %i %i %i %i %i %f 0 %f %i\n", niter, (int)nevts, (int)ntrks, bsize,
              bsize ? (int)(ntrks / bsize) : 0, wall_s, setup_s, nthreads);
  std::fflush(stdout);
}

}  // extern "C"
