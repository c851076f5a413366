// p2z_main.cpp -- command-line driver with the reference executable's output
// (src/propagate-toz-test_OMP.cpp:684-883): it prepares the inputs with the
// reference's generator, runs the hot path through libp2z's C ABI from host
// memory (the reference GPU build's include_data mode), and prints the
// reference's lines -- including the "formatted" line its tools parse and the
// validation block -- so the reference's scripts can drive it unchanged.
//
// usage: p2z_main [SEEDFILE [nevts ntrks bsize nlayer niter [smear [cov_scale]]]]
// SEEDFILE: first line 6 track parameters, 21 covariance elements and the
// charge; then one line per layer with 3 hit positions and 6 covariance
// elements (layer order).  Without arguments -- as the reference's tools run
// its executables, whose seed is compiled in (tools/compare.sh) -- the seed
// file is $P2Z_SEED_FILE, else the reference's known-answer seed in the
// repository beside this executable (../tests/golden/kat_seed.txt), with the
// reference's default sizes.  The environment variable P2Z_FLAGS (an integer,
// decimal or 0x-hex) sets p2z_config.flags, e.g. P2Z_FLAGS=0x20 for the
// reference's own rounding (P2Z_FLAG_REFERENCE_ROUNDING); P2Z_UPDATE selects the
// update kind (p2z_update_kind, default 0 = KalmanUpdate_v2).
#include <sys/time.h>
#include <unistd.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "p2z.h"

static long now_ms() {
  struct timeval tv;
  gettimeofday(&tv, nullptr);
  return (long)tv.tv_sec * 1000 + (long)tv.tv_usec / 1000;
}

// The seed file when none is given: $P2Z_SEED_FILE, else the known-answer
// seed of the repository this executable was built in.
static std::string default_seed_file() {
  if (const char *e = std::getenv("P2Z_SEED_FILE")) return e;
  char exe[4096];
  const ssize_t n = readlink("/proc/self/exe", exe, sizeof exe - 1);
  if (n <= 0) return "tests/golden/kat_seed.txt";
  exe[n] = 0;
  std::string dir(exe);
  dir = dir.substr(0, dir.find_last_of('/'));
  return dir + "/../tests/golden/kat_seed.txt";
}

int main(int argc, char **argv) {
  if (argc > 1 && (std::string(argv[1]) == "-h" || std::string(argv[1]) == "--help")) {
    std::fprintf(stderr, "usage: %s [SEEDFILE [nevts ntrks bsize nlayer niter [smear [cov_scale]]]]\n", argv[0]);
    return 2;
  }
  const std::string seed_file = argc > 1 ? std::string(argv[1]) : default_seed_file();
  long nevts = argc > 2 ? std::atol(argv[2]) : 100;
  long ntrks = argc > 3 ? std::atol(argv[3]) : 9600;
  int bsize = argc > 4 ? std::atoi(argv[4]) : 32;
  int nlayer = argc > 5 ? std::atoi(argv[5]) : 20;
  int niter = argc > 6 ? std::atoi(argv[6]) : 5;
  double smear = argc > 7 ? std::atof(argv[7]) : 1e-7;
  double cov_scale = argc > 8 ? std::atof(argv[8]) : 100.0;

  FILE *f = std::fopen(seed_file.c_str(), "r");
  if (!f) {
    std::fprintf(stderr, "cannot open %s\n", seed_file.c_str());
    return 2;
  }
  p2z_atrk trk;
  for (float &v : trk.par)
    if (std::fscanf(f, "%f", &v) != 1) return 2;
  for (float &v : trk.cov)
    if (std::fscanf(f, "%f", &v) != 1) return 2;
  if (std::fscanf(f, "%d", &trk.q) != 1) return 2;
  std::vector<p2z_ahit> hits;
  for (;;) {
    p2z_ahit h;
    int n = 0;
    for (float &v : h.pos) n += std::fscanf(f, "%f", &v) == 1;
    for (float &v : h.cov) n += std::fscanf(f, "%f", &v) == 1;
    if (n != 9) break;
    hits.push_back(h);
  }
  std::fclose(f);
  if ((int)hits.size() < nlayer) {
    std::fprintf(stderr, "seed file has %zu hits < nlayer %d\n", hits.size(), nlayer);
    return 1;  // the reference exits(1) here (:271-274)
  }

  std::printf("bsize: %d, nb:%d, device: B200 (libp2z)\n", bsize, (int)(ntrks / bsize));
  std::printf("track in pos: x=%f, y=%f, z=%f, r=%f, pt=%f, phi=%f, theta=%f \n", trk.par[0], trk.par[1], trk.par[2],
              sqrtf(trk.par[0] * trk.par[0] + trk.par[1] * trk.par[1]), 1. / trk.par[3], trk.par[4], trk.par[5]);
  std::printf("track in cov: %.2e, %.2e, %.2e \n", trk.cov[0], trk.cov[2], trk.cov[5]);
  for (int lay = 0; lay < nlayer; lay++)
    std::printf("hit in layer=%d, pos: x=%f, y=%f, z=%f, r=%f \n", lay, hits[lay].pos[0], hits[lay].pos[1],
                hits[lay].pos[2], sqrtf(hits[lay].pos[0] * hits[lay].pos[0] + hits[lay].pos[1] * hits[lay].pos[1]));
  std::printf("produce nevts=%li ntrks=%li smearing by=%2.1e \n", nevts, ntrks, smear);
  std::printf("NITER=%d\n", niter);

  const long setup_start = now_ms();
  p2z_config cfg = {};
  cfg.abi_version = P2Z_ABI_VERSION;
  cfg.bsize = bsize;
  cfg.nevts = nevts;
  cfg.ntrks = ntrks;
  cfg.nlayer = nlayer;
  cfg.niter = niter;
  if (const char *fl = std::getenv("P2Z_FLAGS")) cfg.flags = (uint32_t)std::strtoul(fl, nullptr, 0);
  if (const char *up = std::getenv("P2Z_UPDATE")) cfg.update = (int32_t)std::strtol(up, nullptr, 0);
  const int64_t nb = p2z_num_batches(&cfg);
  if (nb < 0) {
    std::fprintf(stderr, "bad sizes: %s\n", p2z_last_error(nullptr));
    return 2;
  }
  void *h_trk = nullptr, *h_hit = nullptr, *h_out = nullptr;
  if (p2z_host_alloc(&h_trk, p2z_sizeof_mptrk(bsize) * nb) || p2z_host_alloc(&h_hit, p2z_sizeof_mphit(bsize) * nb * nlayer) ||
      p2z_host_alloc(&h_out, p2z_sizeof_mptrk(bsize) * nb)) {
    std::fprintf(stderr, "host allocation failed: %s\n", p2z_last_error(nullptr));
    return 1;
  }
  p2z_status st = p2z_prepare(&trk, hits.data(), (int)hits.size(), bsize, nevts, ntrks, nlayer, smear, cov_scale, h_trk, h_hit);
  if (st != P2Z_OK) {
    std::fprintf(stderr, "p2z_prepare: %s\n", p2z_status_string(st));
    return 1;
  }
  p2z_context *ctx = nullptr;
  if ((st = p2z_create(0, &ctx)) != P2Z_OK) {
    std::fprintf(stderr, "p2z_create: %s (%s)\n", p2z_status_string(st), p2z_last_error(nullptr));
    return 1;
  }
  const long setup_stop = now_ms();
  std::printf("done preparing!\n");

  p2z_stats stats;
  const auto wall_start = std::chrono::high_resolution_clock::now();
  st = p2z_run(ctx, &cfg, h_trk, h_hit, nullptr, h_out, &stats);
  const auto wall_stop = std::chrono::high_resolution_clock::now();
  if (st != P2Z_OK) {
    std::fprintf(stderr, "p2z_run: %s (%s)\n", p2z_status_string(st), p2z_last_error(ctx));
    return 1;
  }
  const double wall = std::chrono::duration_cast<std::chrono::microseconds>(wall_stop - wall_start).count() / 1e6;
  std::printf("setup time time=%f (s)\n", (setup_stop - setup_start) * 0.001);
  std::printf("done ntracks=%li tot time=%f (s) time/trk=%e (s)\n", nevts * ntrks * niter, wall,
              wall / ((double)nevts * ntrks * niter));
  p2z_print_formatted(niter, nevts, ntrks, bsize, wall, (setup_stop - setup_start) * 0.001, 1);
  p2z_validation v;
  p2z_validate(h_out, bsize, nevts, ntrks, hits[nlayer - 1].pos, &v);
  p2z_print_validation(&v);
  p2z_destroy(ctx);
  p2z_host_free(h_trk);
  p2z_host_free(h_hit);
  p2z_host_free(h_out);
  return 0;
}
