/* The C ABI used the way a maintainer adds it to the reference's OpenMP
 * source: the reference's size macros (src/propagate-toz-test_OMP.cpp:18-41,
 * :295) are defined first, the header is included after them, and the config
 * is filled with p2z_config_init from those macros.  Plain C (the header is a
 * C header); compiled and run on the CPU by tests/test_host.py.  Prints the
 * config's fields, one per line. */
#include <stdio.h>

#define nevts 100
#ifndef bsize
#define bsize 32
#endif
#define ntrks 9600
#define nb (ntrks / bsize)
#define smear 0.0000001
#define NITER 5
#define nlayer 20
#define nthreads 64
#define N bsize

#include "p2z.h"

int main(void) {
  p2z_config cfg;
  if (p2z_config_init(&cfg, bsize, nevts, ntrks, nlayer) != P2Z_OK) return 1;
  cfg.niter = NITER;
  cfg.update = P2Z_UPDATE_V2;
  cfg.flags = 0;
  /* the macros are the reference's again after the header */
  if (nb != ntrks / bsize || N != bsize || nthreads != 64 || smear != 0.0000001) return 2;
  printf("abi_version %d\n", (int)cfg.abi_version);
  /* reading the size members back needs the macros out of the way */
#pragma push_macro("bsize")
#pragma push_macro("nevts")
#pragma push_macro("ntrks")
#pragma push_macro("nlayer")
#undef bsize
#undef nevts
#undef ntrks
#undef nlayer
  printf("sizes %d %lld %lld %d\n", (int)cfg.bsize, (long long)cfg.nevts, (long long)cfg.ntrks, (int)cfg.nlayer);
#pragma pop_macro("nlayer")
#pragma pop_macro("ntrks")
#pragma pop_macro("nevts")
#pragma pop_macro("bsize")
  printf("niter %d update %d schedule %d block %d flags %u layout %d tpt %d kfact %g event_ntrks %d\n",
         (int)cfg.niter, (int)cfg.update, (int)cfg.schedule, (int)cfg.block_threads, (unsigned)cfg.flags,
         (int)cfg.layout, (int)cfg.threads_per_track, (double)cfg.kfact, cfg.event_ntrks != NULL);
  printf("batches %lld\n", (long long)p2z_num_batches(&cfg));
  return p2z_config_init(NULL, bsize, nevts, ntrks, nlayer) == P2Z_BAD_ARG ? 0 : 3;
}
