// Host-side launch engine shared by the single-graph and batched entry points.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "enum_launch.h"
#include "internal.h"

namespace gmbe {

// Engine workspace, one per device, shared by every graph and batch on that
// device and reused across calls (grown on demand).  A call holds the
// device's workspace for its whole duration.
struct Workspace {
  std::mutex mu;
  int32_t* scratch = nullptr;
  size_t scratch_bytes = 0;
  EnumCtl* ctl = nullptr;
  Task* q_tasks = nullptr;
  unsigned long long* q_seq = nullptr;
  int32_t q_cap = 0;
  unsigned long long* exit_ns = nullptr;
  int32_t exit_cap = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int32_t* slots = nullptr;  // exported bitmap sub-problems
  uint32_t* slot_bits = nullptr;
  int32_t nslot = 0;
  int32_t* big_slots = nullptr;  // large ones (kBigSlotWords words each)
  uint32_t* big_slot_bits = nullptr;
  int32_t nbig_slot = 0;
  // Single-graph launch descriptors.
  DevGraph* d_graph1 = nullptr;
  long long* d_prefix1 = nullptr;
  unsigned long long* d_gres1 = nullptr;
  // Layout the per-warp count maps were last cleared for (big tier: the
  // first map_big warps, pitch map_big_pitch).
  int64_t map_pitch_words = -1, map_words = -1;
  int32_t map_warps = -1;
  int64_t map_big_pitch = 0;
  int32_t map_big = 0;
  // Two-tier launches: the big-root list and the per-root flags.
  int32_t* big_roots = nullptr;
  uint8_t* big_flag = nullptr;
  size_t big_roots_cap = 0, big_flag_cap = 0;
  int32_t* big_parts = nullptr;  // part records of big roots (4 int32 each)
  size_t big_parts_cap = 0;
  // Persisting L2 of the device (bytes; -1 = not queried yet, 0 = none).
  long long l2_persist = -1;
  int l2_max_window = 0;
  // Bumped whenever a buffer above is (re)allocated: a captured launch that
  // refers to an older generation must be captured again.
  uint64_t gen = 1;
};

Workspace& workspace(int device);

}  // namespace gmbe

// A graph handle (include/mbe.h): the internal graph on the host and device.
struct mbe_graph {
  gmbe::HostGraph h;  // built on the device: sizes, degrees and v_orig/u_orig only
  mbe_opts opts;
  int device = 0;
  bool device_built = false;  // host CSR arrays are fetched when needed (emission)
  int32_t* d_row_off = nullptr;
  int32_t* d_col = nullptr;
  int32_t* d_rev_off = nullptr;
  int32_t* d_rev_col = nullptr;
  uint64_t* d_ukey = nullptr;
  uint64_t* d_vkey = nullptr;
  // Capacities derived from the graph (max over roots).
  int32_t capS = 0, capL = 0;
};

namespace gmbe {

// Builds g's internal graph on its device from an .adj-shaped host CSR (the
// -t swap, -o 0/1/2 ordering, both CSRs, hash keys, capacities); fills the
// host fields sizes, degrees, swapped, v_orig, u_orig.
int device_build_graph(mbe_graph* g, const int32_t* row_off, const int32_t* col, int32_t nV,
                       int32_t nU, int64_t nE);

// Fetches the host CSR copies of a graph built on the device (no-op otherwise).
int ensure_host_csr(mbe_graph* g);

// What one launch needs from the workspace: the largest internal V side (the
// count maps) and the per-warp capacities, maxima over the launch's graphs.
struct LaunchSpec {
  int device = 0;
  int32_t map_words = 1;
  int32_t capC = 1, capL = 1, capS = 1;
  int32_t n_graphs = 1;
  // Two tiers (single-graph launches): n_big warps with these capacities,
  // the others with capC/capL/capS above.  n_big == 0: one tier.
  int32_t n_big = 0;
  int32_t bigC = 1, bigL = 1, bigS = 1;
};

struct LaunchPlan {
  int blocks = 0, warps = 0;
  ScratchLayout sl;
  EnumParams ep;  // ep.n_big_warps / ep.big_sl: the big tier, if any
  SlotPool pool;
  bool clear_maps = false;
  int32_t map_words = 1;
  // Persisting L2 access-policy window of the launch (l2_bytes 0: none).
  const void* l2_base = nullptr;
  size_t l2_bytes = 0;
  float l2_hit = 1.0f;
};

// Device bytes of the scratch of `warps` warps, n_big of them with the big
// layout (n_big == 0: every warp with sl).
inline size_t scratch_bytes(const ScratchLayout& sl, const ScratchLayout& big, int warps,
                            int n_big) {
  return ((size_t)big.words_per_warp * (size_t)n_big +
          (size_t)sl.words_per_warp * (size_t)(warps - n_big)) * sizeof(int32_t);
}

// Allocates or grows the workspace and fixes the launch shape (host-only,
// not capturable).  Caller holds ws.mu.
int engine_prepare(Workspace& ws, const LaunchSpec& spec, const mbe_params& prm, LaunchPlan* plan);

// Resident blocks per SM of the enumeration kernel (the two-tier variant if
// `tiers`) with `smem` bytes of dynamic shared memory per block; also raises
// the kernel's dynamic shared memory limit to `smem` where it is lower.
int enum_blocks_per_sm(bool tiers, size_t smem, int* occ);

// Queues the strided clear of every warp's count map if the layout changed
// since the maps were last cleared (capturable; a no-op otherwise).
int engine_clear_maps(Workspace& ws, LaunchPlan* plan, cudaStream_t st);

// Queues the launch: control-block, ring-tag, slot-map and result clears,
// the count-map clear if the layout changed, and the kernel (capturable).
// ev0/ev1, when given, bracket the kernel.
int engine_enqueue(Workspace& ws, LaunchPlan* plan, const DevGraph* d_graphs,
                   const long long* d_prefix, unsigned long long* d_gres, int n_graphs,
                   cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1);

// Status word -> MBE_ERR_* with a message; clears the count-map state.
int engine_status(Workspace& ws, const EnumCtl& ctl);

// Copies the profile counters of the control block into a result.
void fill_profile(const EnumCtl& ctl, mbe_result* out);

// Root splitting settings of a launch from the parameters.
inline int32_t eager_share_of(const mbe_params& prm) { return prm.eager_share > 0 ? 1 : 0; }

inline void apply_range_split(const mbe_params& prm, int32_t* work, int32_t* chunk) {
  *work = prm.split_mode == 1 ? 0 : std::max(prm.range_split_work, 0);
  *chunk = prm.range_chunk > 0 ? prm.range_chunk : kRangeChunkDefault;
}

// Per-graph tuning fields of a descriptor from parameters.
int apply_tuning(const mbe_params& prm, DevGraph* dg);

// Hash keys (original ids, original sides) of an internal graph.
void host_keys(const HostGraph& h, std::vector<uint64_t>* uk, std::vector<uint64_t>* vk);

// Capacities of a graph: max |N(v)| and max sum_{u in N(v)} d(u) over roots.
int graph_caps(const HostGraph& h, int32_t* capL, int32_t* capS);

// One emitted record (L as internal U ids) -> the biclique in original ids
// and sides, each sorted: R = the common neighbours of L.  R and tmp are
// scratch.
void decode_biclique(const HostGraph& h, std::vector<int32_t>& L, std::vector<int32_t>* us,
                     std::vector<int32_t>* vs, std::vector<int32_t>& R, std::vector<int32_t>& tmp);

}  // namespace gmbe
