// Scratch tiers of one enumeration launch: the host-only decision, kept free
// of CUDA types so that it can be exercised without a device.
#pragma once

#include <cstdint>
#include <vector>

namespace gmbe {

// Per-warp capacities: candidates, |L|, two-hop multiset.
struct TierCaps {
  int32_t capC = 1, capL = 1, capS = 1;
};

struct TierChoice {
  int32_t n_big = 0;       // warps with the big layout (0: one tier)
  int64_t bound = 0;       // two-hop bound of the small tier (two tiers only)
  TierCaps small, big;     // small: every warp when n_big == 0
  uint64_t small_bytes = 0, big_bytes = 0;  // per warp
};

// The launch enumerates n_roots roots; root k is internal vertex roots[k],
// with two-hop multiset S[k] (sum of its neighbours' degrees) and degree D[k].
// nV is the internal V side (the count map), `warps` the launch's warps and
// `budget` the device bytes the scratch may take.
//
// One tier, sized for these roots, when it fits and force_bound <= 0.
// Otherwise two tiers: roots with S > bound (force_bound if > 0, else the
// largest power of two from 2^16 whose small tier takes at most 60 % of the
// budget) are listed in `list` (in the order given) and flagged in `flags`
// (indexed by internal id, nV entries), and force_big warps (0: as many as
// fit, at most half of the warps and at most the listed roots) get the layout
// for the largest root.  The small tier holds any exported sub-problem.
// Returns MBE_OK, MBE_ERR_CAPACITY (a root above 2^30 two-hop entries) or
// MBE_ERR_NOMEM (the small tier or the big warps do not fit).
// pool_for_parts: the listed roots may be split into parts that only big
// warps run, so the big pool is not limited to the number of listed roots
// (as many as fit, at most half of the warps).
int choose_tiers(int32_t nV, int32_t n_roots, const int64_t* S, const int32_t* D,
                 const int32_t* roots, int warps, uint64_t budget, int64_t force_bound,
                 int32_t force_big, TierChoice* out, std::vector<int32_t>* list,
                 std::vector<uint8_t>* flags, bool pool_for_parts = false);

}  // namespace gmbe
