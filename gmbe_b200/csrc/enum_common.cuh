// Device-side types and warp helpers of the enumeration engine.
#pragma once

#include <cstdint>

namespace gmbe {

// Device status codes (negated MBE_ERR_* values are returned by the host).
enum : int32_t {
  kStOk = 0,
  kStTimeout = 1,    // a bounded wait ran out
  kStQueue = 2,      // queue slot never became valid
  kStCapacity = 3,   // a scratch bound was exceeded
  kStDeadline = 4,   // the launch's time limit ran out
};

// Graph in HBM (internal numbering).  rev_* is the U -> V transpose.
struct DevGraph {
  int32_t nV, nU;
  int64_t nE;
  const int32_t* row_off;  // [nV+1]  V -> U
  const int32_t* col;      // [nE]
  const int32_t* rev_off;  // [nU+1]  U -> V
  const int32_t* rev_col;  // [nE]
  const uint64_t* ukey;    // [nU] hash key of internal U vertex (original id, original side)
  const uint64_t* vkey;    // [nV]
  int32_t swapped;         // internal U is the original V side
  // Roots: position p = 0 .. n_roots-1 is internal vertex
  // root_end - 1 - (root_offset + p * root_stride).
  int32_t root_end, root_offset, root_stride, n_roots;
  // Per-graph tuning (results do not depend on it): GMBE's split bounds, the
  // bitmap-tier limit on |L| and the direct-entry limit on |C|.
  int32_t bound_height, bound_size, tier2_max_l, direct_max_c;
};

// A task: up to four internal V vertices, -1 padded (reference LongTask,
// src/GpuUtil.cuh:394-462).  Roots are one-vertex tasks.
struct alignas(16) Task {
  int32_t v[4];
  int32_t graph;  // index into the launch's graph array
  // A root split into `parts` parts (0 = whole): part j pushes, at its first
  // level, only the candidates whose vertex hashes to bucket j.
  int32_t part, parts;
  int32_t pad;
};

// Global control block (one per launch).
struct EnumCtl {
  // results
  unsigned long long count;
  unsigned long long hash;
  unsigned long long non_maximal;
  unsigned long long tasks_split;
  // scheduling
  long long next_root;   // root positions handed out so far (all graphs of the launch)
  int32_t status;        // first error code
  int32_t abort;         // set together with status
  int32_t idle_warps;    // warps waiting for work (export demand)
  int32_t closing;       // serving: the launch is ending (no new roots are claimed)
  unsigned long long pending;   // queued + running tasks (termination)
  unsigned long long q_head;    // next slot to consume
  unsigned long long q_tail;    // next slot to produce
  unsigned long long q_used;    // reserved and not yet consumed slots
  unsigned long long err_info;  // diagnostic of the first error
  // profile counters (summed warp-time in ns, longest task)
  unsigned long long ns_setup, ns_tier1, ns_tier2, ns_idle;
  unsigned long long max_task_ns;   // longest single task
  unsigned long long max_task_info; // (root << 32) | |L| of that task
  unsigned long long max_task_split; // its counts-tier us | bitmap-tier us << 32
  unsigned long long max_task_graph; // its graph
  unsigned long long max_task_pushes; // its pushes: counts tier | bitmap tier << 32
  unsigned long long max_task_shape;  // its |C| | part << 32 | parts << 48 (root tasks)
  unsigned long long n_tasks, n_tier2;
  unsigned long long emit_pos;  // words of biclique records reserved (may pass the buffer's end)
  long long next_big;           // entries of the big-root list handed out so far
  unsigned long long n_big_parts;     // part records appended (may pass big_parts_cap)
  unsigned long long big_parts_head;  // first part record that may have unclaimed parts
};

// Per-warp scratch layout (int32 words unless noted), offsets in words from
// the warp's base.  Built on the host from graph-derived capacities.
struct ScratchLayout {
  int64_t words_per_warp;
  int32_t capC, capL, capS, kmax;
  // offsets
  int64_t map, touched, cv, ncnt, bound, coff, fill, sidx;
  int64_t lv, llevel, lp, aoff, stack, lent;  // lent: entries of each level's L rows
  int64_t lbits;        // counts-tier level bitmaps (kLevelBits x ceil(capC / 32) words)
  int64_t aadj, cadj;
  int64_t masks, sub_v, tcls;  // tcls: class of each touched candidate of a sparse push
  int64_t ckey, ent;           // ckey: hash key per candidate (uint64); ent: packed entries
  int64_t lkey, lmask;  // lkey is uint64 (8-byte aligned offset)
  int64_t lid;          // internal U id of each bitmap-tier L bit (for emission)
  int64_t t2_rec, t2_n, t2_cur, t2_top, r_sum, r_cnt;  // bitmap-tier stack; t2_rec, r_sum uint64
  int64_t act, tlist;
  int32_t act_cap;
  // Words per warp of the first-touch bitmap in shared memory (one bit per
  // V vertex / candidate position); 0 = first touches found by global atomics.
  int32_t seen_words;
  // A first-touch bitmap in global memory (one bit per V vertex / candidate
  // position, gseen_words words), right after the count map: large counting
  // passes without the shared one mark touches with fire-and-forget atomics
  // and collect them by a scan of its words.  Words [0, zero_words) of every
  // warp (count map and this bitmap) are all-zero between tasks.
  int64_t gseen;
  int32_t gseen_words;
  int64_t zero_words;
};

// Slots for bitmap sub-problems handed to idle warps.  Slot s < nslot is
// a regular slot; s >= nslot is large slot s - nslot, for children with more
// candidates than a regular slot holds.
struct SlotPool {
  int32_t* slots;     // nslot x 32768 int32 words
  uint32_t* bits;     // occupancy, nslot / 32 words, zero at launch
  int32_t nslot;      // multiple of 32; 0 disables export
  int32_t nbig;       // large slots: multiple of 32 (0: none)
  int32_t* big;       // nbig x kBigSlotWords int32 words
  uint32_t* big_bits; // their occupancy, nbig / 32 words, zero at launch
  int32_t import_cap; // most candidates any warp of the launch can take in
  int32_t import_l;   // most L vertices any warp can take in
  int32_t import_s;   // largest two-hop multiset any warp can take in
  int32_t pad;
};
constexpr int kBigSlotWords = 1 << 20;  // 4 MiB

// Serving.  Every resident graph is one block of the device arena, aligned to
// 1 << kServeBlockShift bytes and named by its block index: this header, then
// its CSRs and hash keys (the descriptor's pointers point inside the block).
// The host writes the whole block before it publishes the graph; the kernel
// then updates only the counters.  Blocks are bump-allocated and the arena is
// reset only between launches, so no address is rewritten while a launch may
// hold it in a cache.
constexpr int kServeBlockShift = 12;
struct ServeGraph {
  DevGraph g;
  unsigned long long next_root;  // roots claimed (runs past n_roots once exhausted)
  unsigned long long pending;    // roots not yet finished + queued or running children
  unsigned long long res[3];     // count, set hash, non-maximal
  unsigned long long request;    // the host's request id
};

// Completion record, in host-mapped memory; seq = position + 1 once written.
// emit_end: words of biclique records reserved in this launch when the graph
// finished; every record of the graph lies below it (emission only).
struct ServeDone {
  unsigned long long request, count, hash, non_maximal, seq, emit_end;
  unsigned long long pad[2];
};

// Serving state that outlives a launch (device memory).
struct ServeCtl {
  unsigned long long arr_tail;  // graphs published (written by the host)
  unsigned long long arr_head;  // first published graph that may have roots left
  unsigned long long done_pos;  // completion records handed out
  int32_t stop;                 // written by the host: leave at once
  int32_t pad;
};

struct ServeLink {
  ServeCtl* sctl;
  const uint32_t* arr_blk;  // block index of published graph k at k % arr_cap
  ServeDone* done;          // completion ring (host-mapped)
  int32_t arr_cap, done_cap;
  int64_t idle_exit_ns;     // a launch ends after this long with nothing to do
};

struct EnumParams {
  int32_t prune;
  int32_t queue_cap;
  int64_t slot_spin_limit;    // iterations waiting for a claimed slot to be written
  int64_t idle_ns_limit;      // nanoseconds a warp may idle waiting for work
  int64_t time_limit_ns;      // > 0: the launch gives up after this long (kStDeadline)
  int32_t touch_scan;         // 0 auto, 1 always scan the global touch bitmap, -1 never
  int32_t slot_records;       // > 0: regular slots take children of at most this many records
  int32_t share_counts;       // 1: counts-tier children may go to idle warps as vertex lists
  int32_t pad_sc;
  int32_t record_exit;        // -p
  int32_t vertex_split;       // 1: GMBE vertex-tuple child tasks at task set-up
  int32_t n_graphs;           // graphs of this launch (1 for a single enumeration)
  int32_t root_split;         // > 0: a root task with |P|*|L| above this splits into vertex tuples
  int32_t share_min_work;     // |P|*|L| of a child shared out while many warps wait
  int32_t range_work;         // > 0: a root with |P|*|L| above this is split into parts
  int32_t range_chunk;        // P candidates per part
  int32_t eager_share;        // 1: counts-tier children passing the split test always go
  int32_t* emit;              // biclique records [|L|, graph, L ids...], or null
  long long emit_cap;         // words in emit
  const unsigned long long* emit_read;  // ring mode: words the host has consumed (else null)
  int32_t server;             // 1: graphs arrive while the launch runs (ServeLink)
  ServeLink serve;
  // Two scratch tiers (single-graph launches only).  Warps [0, n_big_warps)
  // use big_sl and first take the roots of big_roots (internal ids, in claim
  // order); every other warp uses the launch's layout.  Roots flagged in
  // big_flag (indexed by internal V id) are in that list and are skipped when
  // met through the ordinary root counter.  n_big_warps == 0: one tier.
  int32_t n_big_warps;
  int32_t n_big_roots;
  const int32_t* big_roots;
  const uint8_t* big_flag;
  ScratchLayout big_sl;
  // Parts of listed big roots (only big warps may run them): records of four
  // int32 {root, parts, next part to claim, ready}, all-zero at launch.
  int32_t* big_parts;
  int32_t big_parts_cap;
};

__device__ __forceinline__ uint64_t fmix64(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ULL;
  k ^= k >> 33;
  return k;
}

__device__ __forceinline__ uint64_t biclique_hash(const DevGraph& g, uint64_t sU, uint64_t nU,
                                                  uint64_t sV, uint64_t nV) {
  // Internal U is the L side; the canonical hash takes the original-U side first.
  uint64_t sL = g.swapped ? sV : sU, nL = g.swapped ? nV : nU;
  uint64_t sR = g.swapped ? sU : sV, nR = g.swapped ? nU : nV;
  uint64_t rot = (sR << 29) | (sR >> 35);
  return fmix64(sL ^ rot ^ ((nL << 32) | nR));
}

__device__ __forceinline__ unsigned lane_id() {
  unsigned r;
  asm volatile("mov.u32 %0, %%laneid;" : "=r"(r));
  return r;
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ int warp_min_i(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ int warp_max_i(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Exclusive prefix sum within the warp.
__device__ __forceinline__ int warp_excl_scan(int v, int* total) {
  int lane = (int)lane_id();
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  *total = __shfl_sync(0xffffffffu, x, 31);
  return x - v;
}

// Lower bound: first index in a[0,n) with a[i] >= key.
__device__ __forceinline__ int lower_bound_i(const int32_t* a, int n, int key) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (__ldg(a + mid) < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ bool contains_sorted(const int32_t* a, int n, int key) {
  int p = lower_bound_i(a, n, key);
  return p < n && __ldg(a + p) == key;
}

}  // namespace gmbe
