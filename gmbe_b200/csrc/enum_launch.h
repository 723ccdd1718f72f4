// Host-side launch interface of the enumeration kernel.
#pragma once

#include <cuda_runtime.h>

#include "enum_common.cuh"

namespace gmbe {

#ifndef GMBE_ENUM_WARPS
#define GMBE_ENUM_WARPS 16
#endif
#ifndef GMBE_ENUM_MIN_BLOCKS
#define GMBE_ENUM_MIN_BLOCKS 1
#endif
constexpr int kEnumWarps = GMBE_ENUM_WARPS;    // warps per block
constexpr int kEnumThreads = kEnumWarps * 32;  // threads per block
// Blocks per SM the register allocation is made for (launch bounds).
constexpr int kEnumMinBlocks = GMBE_ENUM_MIN_BLOCKS;
constexpr int kKMax = 4;                       // bitmap words of the tier-2 sub-problem
constexpr int kLevelBits = 8;                  // counts-tier levels with a candidate bitmap

// One persistent launch over p.n_graphs graphs: graphs[i] describes graph i,
// root_prefix[i] counts the roots of graphs before i (root_prefix[n] = all),
// gres[3i .. 3i+2] receives graph i's count, set hash and non-maximal count.
__global__ void mbe_enum_kernel(const DevGraph* graphs, const long long* root_prefix,
                                unsigned long long* gres, const __grid_constant__ EnumParams p,
                                const __grid_constant__ ScratchLayout sl, EnumCtl* ctl,
                                Task* q_tasks, unsigned long long* q_seq, SlotPool pool,
                                int32_t* scratch, unsigned long long* exit_ns);
// The same launch with two scratch tiers (p.n_big_warps > 0): the first
// n_big_warps warps use p.big_sl and take p.big_roots first.
__global__ void mbe_enum_kernel_tiers(const DevGraph* graphs, const long long* root_prefix,
                                      unsigned long long* gres,
                                      const __grid_constant__ EnumParams p,
                                      const __grid_constant__ ScratchLayout sl, EnumCtl* ctl,
                                      Task* q_tasks, unsigned long long* q_seq, SlotPool pool,
                                      int32_t* scratch, unsigned long long* exit_ns);

constexpr int kSlotWordsHost = 32768;  // int32 words per sub-problem slot (128 KiB)
// Most candidate records one slot carries (K = 1): a warp that may run
// another warp's exported sub-problem needs room for this many candidates.
constexpr int32_t kSlotMaxRecords = 8064;
// Largest first-touch bitmap per warp (kEnumWarps of them fit the 227 KiB a block may use).
constexpr int kSeenMaxWords = 3584;
// Dynamic shared memory of a launch with layout sl.
inline size_t enum_smem_bytes(const ScratchLayout& sl) {
  return (size_t)sl.seen_words * sizeof(uint32_t) * kEnumWarps;
}
// |P|*|L| from which a child is shared out while many warps wait for work.
constexpr int32_t kShareMinWorkDefault = 256;
// P candidates per part of a root split into parts.
constexpr int32_t kRangeChunkDefault = 64;
// |P|*|C| above which a root is split into parts unless the caller says
// otherwise (no root of the medium or batched workloads comes near it).
constexpr int32_t kRangeWorkDefault = 1000000000;


// Per-warp scratch layout for the given capacities.
ScratchLayout make_layout(int32_t nV, int32_t capC, int32_t capL, int32_t capS);

}  // namespace gmbe
