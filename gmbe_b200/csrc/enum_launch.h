// Host-side launch interface of the enumeration kernel.
#pragma once

#include <cuda_runtime.h>

#include "enum_common.cuh"

namespace gmbe {

constexpr int kEnumWarps = 16;                 // warps per block
constexpr int kEnumThreads = kEnumWarps * 32;  // threads per block
constexpr int kKMax = 4;                       // bitmap words of the tier-2 sub-problem

__global__ void mbe_enum_kernel(const __grid_constant__ DevGraph g,
                                const __grid_constant__ EnumParams p,
                                const __grid_constant__ ScratchLayout sl, EnumCtl* ctl,
                                Task* q_tasks, unsigned long long* q_seq, SlotPool pool,
                                int32_t* scratch, unsigned long long* exit_ns);

constexpr int kSlotWordsHost = 16384;  // int32 words per sub-problem slot (64 KiB)

// Per-warp scratch layout for the given capacities.
ScratchLayout make_layout(int32_t nV, int32_t capC, int32_t capL, int32_t capS);

}  // namespace gmbe
