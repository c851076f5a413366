// ref_harness.cpp -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// Compiles the reference benchmark's OpenMP source unchanged, from where it
// lies (src/propagate-toz-test_OMP.cpp of the reference tree, found through
// -I), and exposes its functions through a small extern "C" surface so that
// tests and the CPU-baseline leg of bench.py can call the reference itself:
//
//   prepareTracks / prepareHits   src/propagate-toz-test_OMP.cpp:243-293
//   propagateToZ                  src/propagate-toz-test_OMP.cpp:623-682
//   KalmanUpdate_v2               src/propagate-toz-test_OMP.cpp:503-620
//   the timed hot loop            src/propagate-toz-test_OMP.cpp:731-748
//   main (renamed)                src/propagate-toz-test_OMP.cpp:684-883
//
// Sizes (bsize, nevts, ntrks, nlayer, NITER, nthreads) are compile-time macros
// in the reference; oracle/Makefile builds one library per combination it
// needs.  The hot-loop entry below takes the number of events, batches and
// layers at run time and indexes the arrays itself, so one library per bsize
// serves every workload size.
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <math.h>
#include <unistd.h>
#include <sys/time.h>
#include <iostream>
#include <chrono>
#include <iomanip>
#include <vector>
#include <cstring>

#ifdef P2Z_REF_CR_TRIG
// Variant build: the reference's calls to the C library's sinf/cosf are bound
// to correctly rounded versions (a double evaluation rounded once to float).
// glibc's sinf/cosf miss correct rounding in about 0.5-0.8% of arguments; this
// build isolates that single difference from any other.
static inline float p2z_cr_sinf(float x) { return (float)sin((double)x); }
static inline float p2z_cr_cosf(float x) { return (float)cos((double)x); }
#define sinf p2z_cr_sinf
#define cosf p2z_cr_cosf
#endif

#define main p2z_ref_main
#include "propagate-toz-test_OMP.cpp"
#undef main

extern "C" {

int ref_bsize(void) { return bsize; }
int ref_nevts(void) { return nevts; }
int ref_ntrks(void) { return ntrks; }
int ref_nlayer(void) { return nlayer; }
float ref_kfact(void) { return kfact; }
size_t ref_sizeof_mptrk(void) { return sizeof(MPTRK); }
size_t ref_sizeof_mphit(void) { return sizeof(MPHIT); }

// The known-answer seed of the reference: its input track and its 26 hits, in
// the order the reference's main uses them (layer 0 = inputhit25).
void ref_kat_seed(ATRK *trk_out, AHIT *hits_out /* 26 entries */) {
#include "input_track.h"
  *trk_out = inputtrk;
  const AHIT order[26] = {inputhit25, inputhit24, inputhit23, inputhit22, inputhit21, inputhit20, inputhit19,
                          inputhit18, inputhit17, inputhit16, inputhit15, inputhit14, inputhit13, inputhit12,
                          inputhit11, inputhit10, inputhit09, inputhit08, inputhit07, inputhit06, inputhit05,
                          inputhit04, inputhit03, inputhit02, inputhit01, inputhit00};
  for (int i = 0; i < 26; ++i) hits_out[i] = order[i];
}

// srand(1) then the reference's prepareTracks / prepareHits with this
// library's compile-time sizes; copies the results out.  trk_out holds
// nevts*nb MPTRK, hit_out nlayer*nevts*nb MPHIT.
int ref_prepare(const ATRK *seed, const AHIT *hits, int nhits, MPTRK *trk_out, MPHIT *hit_out) {
  if (nhits < nlayer) return 1;  // the reference would exit(1) (:271-274)
  srand(1);
  MPTRK *t = prepareTracks(*seed);
  std::vector<AHIT> hv(hits, hits + nhits);
  MPHIT *h = prepareHits(hv);
  std::memcpy(trk_out, t, sizeof(MPTRK) * (size_t)nevts * nb);
  std::memcpy(hit_out, h, sizeof(MPHIT) * (size_t)nlayer * nevts * nb);
  free(t);
  free(h);
  return 0;
}

// The reference's timed loop (:731-748) over run-time sizes: for every event
// (OpenMP-parallel, as the reference) and batch, copy the input batch to the
// output and apply propagateToZ then KalmanUpdate_v2 for each layer.  Hits
// of batch ib, layer l live at hit[l + nlayer_rt*ib] (bHit, :215-217).
void ref_run(const MPTRK *trk, const MPHIT *hit, MPTRK *out, long nev, long nbev, int nlayer_rt, int nthr) {
  if (nthr > 0) omp_set_num_threads(nthr);
#pragma omp parallel for
  for (long ie = 0; ie < nev; ++ie) {
    for (long ib = 0; ib < nbev; ++ib) {
      const long b = ib + nbev * ie;
      out[b] = trk[b];
      for (int layer = 0; layer < nlayer_rt; ++layer) {
        const MPHIT *bh = &hit[layer + (long)nlayer_rt * b];
        propagateToZ(&out[b].cov, &out[b].par, &out[b].q, &bh->pos, &out[b].cov, &out[b].par);
        KalmanUpdate_v2(&out[b].cov, &out[b].par, &bh->cov, &bh->pos);
      }
    }
  }
}

// Single steps on one batch, for layer-by-layer comparisons.
void ref_propagate_batch(MPTRK *b, const MPHIT *h) {
  propagateToZ(&b->cov, &b->par, &b->q, &h->pos, &b->cov, &b->par);
}
void ref_update_v2_batch(MPTRK *b, const MPHIT *h) { KalmanUpdate_v2(&b->cov, &b->par, &h->cov, &h->pos); }

int ref_main(void) {
  char name[] = "p2z_ref";
  char *argv[] = {name, nullptr};
  int rc = p2z_ref_main(1, argv);
  fflush(stdout);
  return rc;
}

}  // extern "C"
