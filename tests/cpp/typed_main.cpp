// typed_main.cpp -- the reference benchmark's main (src/propagate-toz-test_OMP.cpp:
// 684-883) written against include/p2z_types.hpp: the reference's names and
// call sequence, the B200 library underneath.  Used by the tests to show that
// the typed surface is a drop-in: it reproduces the reference's printed
// validation block.
//
// usage: typed_main SEEDFILE MODE [OUTFILE]
//   SEEDFILE  first line: 6 track parameters, 21 covariance elements, charge;
//             then one line per layer: 3 hit positions, 6 covariance elements
//   MODE      "layers": the reference's loop over layers, calling
//             propagateToZ and KalmanUpdate_v2 on every batch (reference
//             rounding); "run": the fused pass with the reference's rounding;
//             "precise": the fused pass, default (precise) evaluation
//   OUTFILE   optional: the output MPTRK array, raw bytes
// Sizes are macros, as in the reference (-Dbsize=... -Dnevts=... -Dntrks=... -Dnlayer=...).
#ifndef bsize
#define bsize 32
#endif
#ifndef nevts
#define nevts 100
#endif
#ifndef ntrks
#define ntrks 9600
#endif
#ifndef nlayer
#define nlayer 20
#endif
#define nb (ntrks / bsize)

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "p2z_types.hpp"

using ATRK = p2z::ATRK;
using AHIT = p2z::AHIT;
using MPTRK = p2z::MPTRK<bsize>;
using ALLTRKS = p2z::ALLTRKS<bsize>;
using ALLHITS = p2z::ALLHITS<bsize>;

static bool read_seed(const char *path, ATRK &trk, std::vector<AHIT> &hits) {
  FILE *f = std::fopen(path, "r");
  if (!f) return false;
  bool ok = true;
  for (float &v : trk.par) ok &= std::fscanf(f, "%f", &v) == 1;
  for (float &v : trk.cov) ok &= std::fscanf(f, "%f", &v) == 1;
  ok &= std::fscanf(f, "%d", &trk.q) == 1;
  for (;;) {
    AHIT h;
    int n = 0;
    for (float &v : h.pos) n += std::fscanf(f, "%f", &v) == 1;
    for (float &v : h.cov) n += std::fscanf(f, "%f", &v) == 1;
    if (n != 9) break;
    hits.push_back(h);
  }
  std::fclose(f);
  return ok;
}

int main(int argc, char *argv[]) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s SEEDFILE layers|run|precise [OUTFILE]\n", argv[0]);
    return 2;
  }
  ATRK inputtrk;
  std::vector<AHIT> inputhits;
  if (!read_seed(argv[1], inputtrk, inputhits)) return 2;
  const char *mode = argv[2];
  printf("bsize: %d, nb:%d\n", (int)bsize, (int)nb);
  printf("produce nevts=%i ntrks=%i smearing by=%2.1e \n", nevts, ntrks, 1e-7);

  try {
    p2z::RefRandom rng(1);  // srand(1): the C library's initial state
    ALLTRKS trk = p2z::prepareTracks<bsize>(inputtrk, nevts, ntrks, rng);
    ALLHITS hit = p2z::prepareHits<bsize>(inputhits, nevts, ntrks, nlayer, rng);
    ALLTRKS outtrk(nevts, ntrks);
    printf("done preparing!\n");

    p2z::Device dev;
    if (std::strcmp(mode, "layers") == 0) {
      // the reference's loop body, on every batch at once
      p2z::DeviceTracks<bsize> obtracks(dev, trk);
      p2z::DeviceHits<bsize> bhits(dev, hit);
      for (int layer = 0; layer < nlayer; ++layer) {
        p2z::propagateToZ(obtracks, bhits, layer);
        p2z::KalmanUpdate_v2(obtracks, bhits, layer);
      }
      outtrk = obtracks.download();
    } else {
      p2z::RunOptions o;
      if (std::strcmp(mode, "run") == 0) o.flags = P2Z_FLAG_REFERENCE_ROUNDING;
      p2z::run(dev, trk, hit, outtrk, o);
    }

    // a track of the first batch, through the reference's accessors
    const MPTRK *b0 = outtrk.bTk(0, 0);
    printf("track 0: x=%f y=%f z=%f pt=%f phi=%f theta=%f cov(0,0)=%e\n", p2z::x(b0, 0), p2z::y(b0, 0),
           p2z::z(b0, 0), 1.f / p2z::ipt(b0, 0), p2z::phi(b0, 0), p2z::theta(b0, 0), p2z::cov(b0, 0, 0, 0));

    if (argc > 3) {
      FILE *f = std::fopen(argv[3], "wb");
      if (!f || std::fwrite(outtrk.btrks, 1, outtrk.bytes(), f) != outtrk.bytes()) return 3;
      std::fclose(f);
    }
    p2z::print_validation(p2z::validate(outtrk, inputhits[nlayer - 1]));
  } catch (const p2z::Error &e) {
    std::fprintf(stderr, "p2z error: %s\n", e.what());
    return 1;
  }
  return 0;
}
