// mbe_gen: writes one seeded synthetic workload graph as an .adj file, from
// the generator spec given on the command line (the fields of mbe_gen_spec,
// include/mbe.h).  A stand-alone program built from the generator sources
// only (no device code), so that a process that must not load the engine
// (the timed CPU runs of the reference's own enumerators) can still make the
// benchmark's inputs.
//
// usage: mbe_gen <out.adj> nU nV n_edges gamma_u gamma_v max_deg_u max_deg_v seed
//                n_blocks block_u block_v block_p pair_p_max
#include <cstdio>
#include <cstdlib>

#include "mbe.h"

int main(int argc, char** argv) {
  if (argc != 15) {
    fprintf(stderr,
            "usage: %s <out.adj> nU nV n_edges gamma_u gamma_v max_deg_u max_deg_v seed "
            "n_blocks block_u block_v block_p pair_p_max\n",
            argv[0]);
    return 2;
  }
  mbe_gen_spec s = {};
  s.nU = atoll(argv[2]);
  s.nV = atoll(argv[3]);
  s.n_edges = atoll(argv[4]);
  s.gamma_u = atof(argv[5]);
  s.gamma_v = atof(argv[6]);
  s.max_deg_u = atoll(argv[7]);
  s.max_deg_v = atoll(argv[8]);
  s.seed = strtoull(argv[9], nullptr, 10);
  s.n_blocks = atoi(argv[10]);
  s.block_u = atoi(argv[11]);
  s.block_v = atoi(argv[12]);
  s.block_p = atof(argv[13]);
  s.pair_p_max = atof(argv[14]);
  int32_t *ro = nullptr, *col = nullptr, nV = 0, nU = 0;
  int64_t nE = 0;
  int rc = mbe_gen_chung_lu(&s, &ro, &col, &nV, &nU, &nE);
  if (rc == MBE_OK) rc = mbe_write_adj(argv[1], ro, col, nV);
  if (rc != MBE_OK) {
    fprintf(stderr, "mbe_gen: %s\n", mbe_last_error_string());
    return 1;
  }
  printf("%d %d %lld\n", nV, nU, (long long)nE);
  mbe_free(ro);
  mbe_free(col);
  return 0;
}
