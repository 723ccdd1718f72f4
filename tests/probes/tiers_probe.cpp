// Runs gmbe::choose_tiers on a request read from a file and prints the
// decision, for the CPU tests of the scratch-tier plan (no device needed).
// Input (little-endian): int32 nV, int32 n_roots, int32 warps, int32 force_big,
// uint64 budget, int64 force_bound, then int64 S[n], int32 D[n], int32 roots[n].
#include <cstdint>
#include <cstdio>
#include <vector>

#include "tiers.h"

int main(int argc, char** argv) {
  if (argc != 2) return 2;
  FILE* f = fopen(argv[1], "rb");
  if (!f) return 2;
  int32_t hdr[4];
  uint64_t budget;
  int64_t force_bound;
  if (fread(hdr, sizeof(hdr), 1, f) != 1 || fread(&budget, 8, 1, f) != 1 ||
      fread(&force_bound, 8, 1, f) != 1)
    return 2;
  const int32_t nV = hdr[0], n = hdr[1], warps = hdr[2], force_big = hdr[3];
  std::vector<int64_t> S(n);
  std::vector<int32_t> D(n), roots(n);
  if ((n && fread(S.data(), 8, n, f) != (size_t)n) || (n && fread(D.data(), 4, n, f) != (size_t)n) ||
      (n && fread(roots.data(), 4, n, f) != (size_t)n))
    return 2;
  fclose(f);
  gmbe::TierChoice ch;
  std::vector<int32_t> list;
  std::vector<uint8_t> flags;
  const int rc = gmbe::choose_tiers(nV, n, S.data(), D.data(), roots.data(), warps, budget,
                                    force_bound, force_big, &ch, &list, &flags);
  long long flagged = 0, mismatch = 0;
  for (uint8_t x : flags) flagged += x;
  for (int32_t v : list) mismatch += (v < 0 || v >= (int32_t)flags.size() || !flags[v]);
  printf("rc %d\nn_big %d\nbound %lld\n", rc, ch.n_big, (long long)ch.bound);
  printf("small %d %d %d\nbig %d %d %d\n", ch.small.capC, ch.small.capL, ch.small.capS,
         ch.big.capC, ch.big.capL, ch.big.capS);
  printf("small_bytes %llu\nbig_bytes %llu\n", (unsigned long long)ch.small_bytes,
         (unsigned long long)ch.big_bytes);
  printf("list %zu\nflagged %lld\nmismatch %lld\n", list.size(), flagged, mismatch);
  printf("first %d\nlast %d\n", list.empty() ? -1 : list.front(), list.empty() ? -1 : list.back());
  return 0;
}
