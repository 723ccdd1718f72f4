/*
 * mbe.h -- C ABI of the B200 maximal biclique enumeration (MBE) engine.
 *
 * This is the drop-in boundary for the single-GPU GMBE hot path
 * (`MBE_GPU -s 2`).  The reference exposes that path only as C++ classes:
 *   - CSRBiGraph::Read / CopyToGpu / Reset      (src/BiGraph.h:23-38, src/BiGraph.cu:13-278, 413-454)
 *   - IterFinderGpu6(graph, bound_height, bound_size), Execute()   (src/IterFinderGpu.h:77-90,
 *     src/IterFinderGpu.cu:1056-1119)
 *   - BicliqueFinder::PrintResult                 (src/BicliqueFinder.cu:9-16)
 * Every entry point below names the reference interface it replaces.  The C++
 * classes with the reference's names (CSRBiGraph, IterFinderGpu6, ...) are
 * provided on top of this ABI by include/mbe_finder.h.
 *
 * Conventions
 *   - Every function returns an int status: MBE_OK (0) or a negative MBE_ERR_*.
 *     The reference exits the process on any CUDA error (gpuErrchk,
 *     src/Utility.h:30-39); this ABI reports instead, and mbe_last_error_string()
 *     gives the message of the calling thread's last failure.
 *   - Plain pointers and sizes only.  Vertex ids are int32, edge counts int64,
 *     counters uint64 (the reference's `int maximal_nodes_` wraps past 2^31).
 *   - A graph handle owns host and device copies of the CSR.  One handle may be
 *     used by one host thread at a time.
 *
 * Biclique identity and the set hash
 *   A maximal biclique is (L, R), L a set of U ids (the integers on an .adj
 *   line), R a set of V ids (0-based .adj line numbers), L = N(R), R = N(L),
 *   both non-empty.  Ids are always the ORIGINAL input ids, whatever side swap
 *   (-t) or row ordering (-o) was applied internally.  The set hash is
 *     key_U(u) = fmix64(2u), key_V(v) = fmix64(2v+1)      (MurmurHash3 fmix64)
 *     sL = sum key_U(u), sR = sum key_V(v)                 (mod 2^64)
 *     H(L,R) = fmix64(sL ^ rotl64(sR,29) ^ (|L|<<32 | |R|))
 *     set_hash = sum over all maximal bicliques of H      (mod 2^64)
 */
#ifndef GMBE_B200_MBE_H
#define GMBE_B200_MBE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define MBE_OK 0
#define MBE_ERR_INVALID (-1)    /* bad argument */
#define MBE_ERR_IO (-2)         /* file cannot be opened or read */
#define MBE_ERR_FORMAT (-3)     /* .adj row not ascending/unique, empty row, bad token, id >= 2^31 */
#define MBE_ERR_CUDA (-4)       /* CUDA runtime error */
#define MBE_ERR_NOMEM (-5)      /* host or device allocation failed */
#define MBE_ERR_TIMEOUT (-6)    /* a bounded device wait ran out */
#define MBE_ERR_QUEUE_FULL (-7) /* device worklist capacity exceeded */
#define MBE_ERR_CAPACITY (-8)   /* a per-warp scratch bound was exceeded */
#define MBE_ERR_ADMISSION (-9)  /* serving: request can never fit the arena */
#define MBE_ERR_CANCELLED (-10) /* serving: request cancelled */
#define MBE_ERR_NOT_FOUND (-11) /* serving: unknown request id */
#define MBE_ERR_AGAIN (-12)     /* serving: result not ready yet */

/* ---- options (reference: struct Option, src/BiGraph.h:13-22) ------------ */
typedef struct mbe_opts {
  int32_t uvtrans;   /* -t: 0 keep sides; 1 make V the smaller side; 2 the larger */
  int32_t order;     /* -o: 0 input order; 1 V rows by (size asc, lexicographic); 2 size desc */
  int32_t fast_mode; /* -f: 1 skips the two-hop degree statistics */
  int32_t device;    /* CUDA device ordinal (the reference always uses device 0) */
} mbe_opts;

/* ---- graph summary (reference: CSRBiGraph fields, src/BiGraph.h:30) ---- */
typedef struct mbe_graph_info {
  int32_t U_size, V_size;  /* internal sides, after the -t swap */
  int64_t edge_size;
  int32_t U_degree, V_degree;   /* max degrees */
  int32_t U_2degree, V_2degree; /* max two-hop degrees (0 under fast_mode) */
  int32_t swapped;              /* 1 if -t swapped U and V */
} mbe_graph_info;

/* ---- enumeration parameters (reference: IterFinderGpu6 ctor args and the
 *      compile-time switches PRUNE_EN / WARP_PER_BLOCK, src/CMakeLists.txt) */
typedef struct mbe_params {
  int32_t bound_height;    /* -m (default 20): a task is split when (|P| > h or |L| > h) ... */
  int32_t bound_size;      /* -n (default 1500): ... and |P|*|L| > bound_size (|P| = C - next) */
  int32_t prune;           /* 1 = pro-active pruning (PRUNE_EN, default), 0 = off */
  int32_t blocks;          /* persistent grid size, 0 = SM count x occupancy */
  int32_t queue_capacity;  /* split-task ring entries, 0 = sized from the graph */
  int32_t bitmap_max_l;    /* bitmap tier for |L| <= this (<= 128); 0 = 128; -1 = counts tier only */
  int64_t wait_limit_ns;   /* longest a warp may idle waiting for work, 0 = 600 s */
  int32_t sm_timing;       /* -p: record each block's exit time */
  int32_t root_begin;      /* enumerate only roots [root_begin, root_end) of the internal */
  int32_t root_end;        /*   order (0, 0 = all); the internal order is -t/-o applied   */
  int32_t shard_count;     /* 0/1 = every root of the range; n > 1 = only the roots at     */
  int32_t shard_index;     /*   positions p = shard_index mod n, counted from the top      */
  int32_t split_mode;      /* how a task passing the split test is shared out:             */
                           /*   0 = its children's bitmap sub-problems go to idle warps     */
                           /*   1 = GMBE's vertex-tuple child tasks (src/IterFinderGpu.cu:835-910) */
  int32_t direct_max_c;    /* a task with |L| <= bitmap_max_l goes straight to the bitmap  */
                           /*   tier only while |C| <= this (0 = 16384); larger candidate  */
                           /*   sets go through the counts tier's sparse pushes            */
  int32_t root_split_size; /* split_mode 0: a root task (one vertex) with |P|*|L| above    */
                           /*   this is split into GMBE's vertex-tuple child tasks, so a   */
                           /*   heavy root's first level runs on many warps; deeper levels */
                           /*   still share out sub-problems.  <= 0 = never (default)      */
  int32_t share_min_work;  /* split_mode 0: while over an eighth of the warps wait for    */
                           /*   work, any child with |P|*|L| >= this is shared out, beyond */
                           /*   the split test's children (0 = default: 256)               */
  int32_t range_split_work; /* split_mode 0: a maximal root with |P|*|C| above this is   */
                           /*   split into parts of range_chunk P candidates; each part  */
                           /*   redoes the root's set-up and pushes, at the first level, */
                           /*   only the candidates whose id hashes to it (earlier parts */
                           /*   act as Q).  0 = default, 10^9; < 0 = never.  In a       */
                           /*   launch with two scratch tiers a listed big root's parts  */
                           /*   run on the big warps only                                */
  int32_t range_chunk;     /* P candidates per part (0 = default 64)                     */
  int32_t eager_share;     /* split_mode 0: a child of the counts tier (|L| > bitmap_max_l) */
                           /*   that passes the split test is shared out even while no  */
                           /*   warp waits: 1 = yes, <= 0 = no (default)                */
  int32_t big_two_hop;     /* mbe_enumerate with two scratch tiers: roots whose two-hop   */
                           /*   multiset (sum of their neighbours' degrees) exceeds this  */
                           /*   run on a pool of warps sized for the largest root; the    */
                           /*   other warps are sized for this bound.  0 = two tiers only */
                           /*   when one layout for every warp does not fit the device    */
                           /*   (the bound is then chosen); needs split_mode 0, and turns */
                           /*   root_split_size off                                       */
  int32_t big_warps;       /* warps of that pool (0 = as many as fit, at most half)      */
  int32_t l2_window;       /* 0 = default: the launch keeps the graph's U -> V lists in a  */
                           /*   persisting L2 access-policy window (as much as the       */
                           /*   device's persisting L2 holds); < 0 = no window            */
  int64_t time_limit_ns;   /* a launch that runs longer than this gives up: every warp    */
                           /*   leaves at its next check (task boundary, counts-tier step,*/
                           /*   or every 4,096 bitmap-tier steps) and the call returns    */
                           /*   MBE_ERR_TIMEOUT; the result is then incomplete.  0 = none */
  int32_t touch_scan;      /* how counting passes find first touches when the per-warp    */
                           /*   shared-memory bitmap does not fit (|V| above ~114k):      */
                           /*   0 = default: a large pass sets bits in a global bitmap    */
                           /*   with fire-and-forget atomics and scans it, a small one    */
                           /*   waits for each atomic's old value; 1 = every pass scans,  */
                           /*   with the shared bitmap off; -1 = never scan.  Results do  */
                           /*   not depend on it                                          */
  int32_t slot_records;    /* a shared-out child with more candidates than this (0 =     */
                           /*   as many as a 128 KiB slot holds) goes through a 4 MiB     */
                           /*   slot instead; results do not depend on it                 */
  int32_t share_counts;    /* counts-tier children (|L| above the bitmap tier) go to      */
                           /*   idle warps as vertex lists: 0 = default, yes; < 0 = no     */
  int32_t reserved_r;      /* zero */
} mbe_params;

typedef struct mbe_result {
  uint64_t count;        /* number of maximal bicliques */
  uint64_t set_hash;     /* order-independent canonical set hash (see above) */
  uint64_t non_maximal;  /* branches rejected by the maximality check */
  uint64_t tasks_split;  /* tasks expanded through the split queue */
  double enum_seconds;   /* host wall time of mbe_enumerate (reference: exe_time_) */
  float kernel_ms;       /* CUDA-event time of the enumeration kernel(s) */
  int32_t status;        /* device status word (0 = OK) */
  double sm_exit_max_ms; /* -p: latest time a block finished its last task, ms after launch */
  double sm_exit_min_ms; /* -p: earliest such time (max - min = load-balance skew) */
  double warp_busy_frac; /* -p: share of warp-time spent inside tasks */
  /* Summed warp-time (ms) by phase: task set-up, counts tier, bitmap tier,
   * idle waiting; the longest single task (ms), its root (internal id) and
   * that root's |N(v)|; tasks run and bitmap sub-problems solved. */
  double setup_ms, tier1_ms, tier2_ms, idle_ms, max_task_ms;
  int32_t max_task_root, max_task_degree;
  uint64_t n_tasks, n_subproblems;
  /* The longest task's time in the counts and bitmap tiers, and its graph
   * (the launch's graph index: descriptor order in a batch). */
  double max_task_tier1_ms, max_task_tier2_ms;
  int32_t max_task_graph, reserved;
  /* The longest task's pushes in the counts and bitmap tiers, its |C| and,
   * for a root split into parts, its part and the number of parts. */
  uint64_t max_task_pushes1, max_task_pushes2;
  int32_t max_task_cands, max_task_part, max_task_parts, reserved2;
} mbe_result;

/* Default parameters: bound_height 20, bound_size 1500, prune 1. */
void mbe_params_default(mbe_params* p);
void mbe_opts_default(mbe_opts* o);

/* ---- graph lifetime ----------------------------------------------------- */
typedef struct mbe_graph mbe_graph;

/* Parse an .adj file and upload it.  Replaces CSRBiGraph::Read
 * (src/BiGraph.cu:13-278) followed by CopyToGpu (src/BiGraph.cu:413-431).
 * Unlike the reference, a row that is not strictly ascending, an empty row
 * or an id >= 2^31-1 is reported as MBE_ERR_FORMAT, and a missing file as
 * MBE_ERR_IO (the reference prints "Can't open file" and continues with an
 * empty graph). */
int mbe_graph_from_adj(const char* path, const mbe_opts* opts, mbe_graph** out);

/* Build a graph from an .adj-shaped CSR in host memory: row v (0..nV-1) holds
 * the U ids col[row_off[v] .. row_off[v+1]).  nU = 0 means max id + 1, as the
 * reference computes U_size (src/BiGraph.cu:31).  Same checks as above.
 * Replaces the in-memory half of CSRBiGraph::Read plus CopyToGpu. */
int mbe_graph_from_csr(const int32_t* row_off, const int32_t* col, int32_t nV, int32_t nU,
                       int64_t nE, const mbe_opts* opts, mbe_graph** out);

/* Same input, checks and result as mbe_graph_from_csr, with the build on the
 * device: the input CSR is uploaded once and the transposes, the -t swap, the
 * -o 1/2 degree ordering, the hash keys and the capacities are computed there
 * (no reference counterpart; the reference builds on the host in
 * CSRBiGraph::Read, src/BiGraph.cu:13-278).  Rows of equal degree keep their
 * input order instead of the reference's lexicographic tie-break; the set of
 * maximal bicliques (count and set hash) is the same.  Without fast_mode the
 * two-hop statistics are host work, and the call builds as
 * mbe_graph_from_csr does.  nV = 0 or nE = 0 is MBE_ERR_INVALID here. */
int mbe_graph_build_on_device(const int32_t* row_off, const int32_t* col, int32_t nV, int32_t nU,
                              int64_t nE, const mbe_opts* opts, mbe_graph** out);

int mbe_graph_get_info(const mbe_graph* g, mbe_graph_info* info);

/* Release host and device memory.  Replaces CSRBiGraph::Reset (src/BiGraph.cu:433-454). */
int mbe_graph_free(mbe_graph* g);

/* Release the device memory the library keeps on `device` between calls of
 * mbe_enumerate and of batches (per-warp scratch, split ring, export slots;
 * on the largest graphs most of the device).  The next call allocates again.
 * The reference allocates and frees per finder object
 * (src/IterFinderGpu.cu:1056-1093); this engine caches, and this call is how
 * a caller hands the memory back, e.g. before another process uses the GPU. */
int mbe_device_release(int32_t device);

/* ---- enumeration --------------------------------------------------------- */
/* Count all maximal bicliques of g and their set hash on g's device.
 * Replaces IterFinderGpu6::IterFinderGpu6 + Execute (src/IterFinderGpu.cu:1056-1119).
 * `params` may be NULL (defaults).  Synchronous on the calling thread. */
int mbe_enumerate(mbe_graph* g, const mbe_params* params, mbe_result* out);

/* As mbe_enumerate, also writing every maximal biclique into buf (no
 * counterpart in the reference, which only counts): records
 * [|U|, |V|, U ids ascending, V ids ascending] in original ids and sides,
 * packed one after another, *used_words in all.  The kernel emits each
 * biclique's L side into a ring the host drains while the launch runs (see
 * mbe_enumerate_emit_stream); the host derives the other side as the common
 * neighbourhood of L.  MBE_ERR_CAPACITY (with the records that fit,
 * *used_words of them) when buf is too small; count and hash stay exact. */
int mbe_enumerate_emit(mbe_graph* g, const mbe_params* params, mbe_result* out, int32_t* buf,
                       int64_t buf_words, int64_t* used_words);

/* One maximal biclique, in original ids and sides, ids ascending; return 0 to
 * go on, non-zero to receive no more (the enumeration still completes and
 * `out` stays exact). */
typedef int (*mbe_emit_fn)(const int32_t* u_ids, int32_t n_u, const int32_t* v_ids, int32_t n_v,
                           void* user);

/* As mbe_enumerate, handing every maximal biclique to `fn` while the launch
 * runs (no counterpart in the reference, whose GPU path only counts; its CPU
 * finders print each biclique at the count site, src/BicliqueFinder.cu:20-57).
 * The kernel writes each biclique's L side into a ring of ring_words int32
 * words in pinned, device-mapped host memory (at least one largest record);
 * this call drains and decodes the ring in the calling thread while the
 * kernel runs, and a producer that would overrun undrained records waits
 * for room.  Any number of bicliques passes through a ring of fixed size.
 * mbe_enumerate_emit is this call with a 2^22-word ring and a callback that
 * fills the caller's buffer. */
int mbe_enumerate_emit_stream(mbe_graph* g, const mbe_params* params, mbe_result* out,
                              int64_t ring_words, mbe_emit_fn fn, void* user);

/* Thread-local message of the last failed call ("" if none). */
const char* mbe_last_error_string(void);

/* Enumeration that allocates nothing.  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc: code inside a framework whose own
 * allocator owns all device memory, code that is recorded into a CUDA graph,
 * or a process whose device-memory budget is fixed up front.  mbe_enumerate
 * allocates (and caches) its workspace; this call instead takes every working
 * buffer from one static device pool of 64 MiB built into the library, which
 * every GPU that loads the library holds until the process exits.
 *
 * Inputs (device memory, owned by the caller), in the engine's numbering with
 * no side swap or reordering, roots = V rows:
 *   d_row_off[nV+1], d_col[nE]   V -> U rows, strictly ascending U ids
 *   d_rev_off[nU+1], d_rev_col[nE] its transpose (U -> V rows, ascending)
 *   max_two_hop   optional bound on sum_{u in N(v)} d(u) over all roots v
 *                 (0 = use nE); a tighter bound lets more warps fit the pool
 *   params        NULL = defaults; sm_timing, queue_capacity, root range,
 *                 shards, split_mode, direct_max_c and the sharing settings
 *                 are ignored: all roots, a fixed 4096-entry split ring, GMBE's
 *                 vertex-tuple children (split_mode 1, as there is no room for
 *                 sub-problem slots), and every task whose |L| fits the bitmap
 *                 tier goes there straight from set-up
 * Output (device memory, owned by the caller): d_out[4] = count, set hash,
 * non-maximal branches, device status (0 = OK, else a device error code).
 * Ids in the hash are the input ids.
 *
 * The work is queued on `stream` (a cudaStream_t; NULL = legacy default
 * stream) and the call returns without waiting: read d_out after the stream
 * completes.  The call fails with MBE_ERR_CAPACITY, before queuing anything,
 * when one 16-warp block's scratch for this graph (roughly
 * 4*(20*nV + 2*max_two_hop) bytes per warp) plus the hash keys do not fit
 * the pool.  The first call on each device looks up the pool's device
 * address with that device current; make that first call before any stream
 * capture.  Every call on a device shares the one pool, which keeps the last
 * call's contents (each call clears what must start at zero): calls whose
 * work overlaps on the GPU race on it and must be serialised by the caller
 * (one stream, or events). */
int mbe_enumerate_device_noalloc(const int32_t* d_row_off, const int32_t* d_col, int32_t nV,
                                 const int32_t* d_rev_off, const int32_t* d_rev_col, int32_t nU,
                                 int64_t nE, int64_t max_two_hop, const mbe_params* params,
                                 unsigned long long* d_out, void* stream);

/* ---- batched enumeration ---------------------------------------------------
 * No counterpart in the reference (it enumerates one graph per process,
 * src/main.cu).  Many graphs in one device arena and one persistent launch,
 * captured in a CUDA graph on the first run and replayed after that. */
typedef struct mbe_batch mbe_batch;

/* Builds a batch from n .adj-shaped host CSRs (graph i: row_offs[i] with
 * nVs[i]+1 entries, cols[i] with nEs[i] entries; nUs may be NULL = max id+1).
 * Each graph gets the same -t/-o treatment as mbe_graph_from_csr. */
int mbe_batch_from_csr(int32_t n, const int32_t* const* row_offs, const int32_t* const* cols,
                       const int32_t* nVs, const int32_t* nUs, const int64_t* nEs,
                       const mbe_opts* opts, mbe_batch** out);
int mbe_batch_size(const mbe_batch* b);

/* Per-graph tuning (bound_height, bound_size, bitmap_max_l, direct_max_c of
 * `p`) for graph `index` (-1 = all).  Results do not depend on it. */
int mbe_batch_set_tuning(mbe_batch* b, int32_t index, const mbe_params* p);
int mbe_batch_get_tuning(const mbe_batch* b, int32_t index, mbe_params* out);

/* Enumerates every graph of the batch in one launch.  `params` supplies the
 * launch-wide settings (pruning, split mode, blocks, queue, wait limit);
 * per_graph (n entries, may be NULL) gets count / set_hash / non_maximal per
 * graph in input order; total (may be NULL) gets the sums, the kernel time
 * and the profile counters. */
int mbe_batch_run(mbe_batch* b, const mbe_params* params, mbe_result* per_graph,
                  mbe_result* total);

/* Chooses per-graph tuning by size class: the graphs are split into
 * n_classes quantiles of estimated work (sum of squared U degrees), and for
 * each class a set of candidate tunings is timed on that class alone; the
 * fastest is kept.  Every candidate must reproduce the same per-graph count
 * and set hash, else MBE_ERR_CUDA.  chosen (n_classes entries, may be NULL)
 * receives the candidate picked per class. */
int mbe_batch_autotune(mbe_batch* b, const mbe_params* params, int32_t n_classes,
                       int32_t* chosen);

int mbe_batch_free(mbe_batch* b);

/* ---- serving ---------------------------------------------------------------
 * No counterpart in the reference.  A server keeps graphs and enumeration
 * state resident on one GPU and feeds them to one persistent launch while it
 * runs (continuous batching): a request submitted while others are on the
 * GPU is admitted as soon as arena memory and a graph slot are free, and its
 * roots are then claimed by the same warps that work on the others.  A launch
 * ends after idle_exit_ns with nothing to do; the server starts another when
 * work arrives.  Per request the count, set hash and non-maximal count are
 * exactly those of mbe_enumerate on the same CSR and options. */
typedef struct mbe_server mbe_server;

typedef struct mbe_server_config {
  int32_t device;
  int32_t max_graphs;   /* graphs admitted and not yet finished (0 = 4096) */
  int64_t arena_bytes;  /* device memory for resident graphs (0 = 1 GiB) */
  /* Per-warp capacities, fixed for the server's life.  A request whose
   * internal V side, largest root degree or largest two-hop multiset of a
   * root exceeds them can never run: mbe_server_submit rejects it with
   * MBE_ERR_ADMISSION.  0 = 32768 / 4096 / 65536. */
  int32_t max_v;
  int32_t max_degree;
  int32_t max_two_hop;
  /* Host threads that prepare submitted graphs (the -t/-o build, hash keys
   * and the arena image) while the GPU runs others (0 = the host's hardware
   * threads, at most 8). */
  int32_t prep_threads;
  int64_t idle_exit_ns; /* a launch ends after this long without work (0 = 200 us) */
} mbe_server_config;

typedef struct mbe_server_stats {
  uint64_t submitted, admitted, completed, rejected, cancelled;
  uint64_t launches;      /* persistent launches so far */
  uint64_t arena_resets;  /* times the arena was rewound (nothing resident, no launch) */
  int64_t resident;       /* admitted, not yet finished */
  int64_t waiting;        /* submitted, not yet admitted */
  int64_t arena_used, arena_bytes;
  /* Progress, for diagnosis: graphs published to the device and completions
   * collected; whether a launch runs; the device's arrival head and tail,
   * completions handed out, and tasks in flight in the current launch. */
  uint64_t published, collected;
  int64_t launch_running;
  uint64_t dev_head, dev_tail, dev_done, dev_pending;
} mbe_server_stats;

void mbe_server_config_default(mbe_server_config* c);

/* `params` (may be NULL = defaults) applies to every request. */
int mbe_server_create(const mbe_server_config* cfg, const mbe_params* params, mbe_server** out);

/* Checks and copies one .adj-shaped CSR and queues it; returns at once with
 * its id.  The capacity checks run here, in the caller's thread (they need
 * only the two sides' degrees: the -o order does not change them); the -t/-o
 * build of `opts`, as in mbe_graph_from_csr, runs on the server's preparation
 * threads.  Admission (arena space and a graph slot) then follows submission
 * order among prepared graphs.  Errors: MBE_ERR_FORMAT / MBE_ERR_INVALID for
 * bad input, MBE_ERR_ADMISSION if the graph exceeds the server's capacities
 * or arena.  enum_seconds of the result counts from this call. */
int mbe_server_submit(mbe_server* s, const int32_t* row_off, const int32_t* col, int32_t nV,
                      int32_t nU, int64_t nE, const mbe_opts* opts, uint64_t* request_id);

/* Result of a finished request (then forgotten): MBE_OK with count, set_hash,
 * non_maximal and enum_seconds = time from submit to result; MBE_ERR_AGAIN
 * if not finished; MBE_ERR_NOT_FOUND for an unknown id; MBE_ERR_CANCELLED for
 * a cancelled one; a launch failure's code for a request it took down. */
int mbe_server_poll(mbe_server* s, uint64_t request_id, mbe_result* out);

/* As mbe_server_poll, waiting up to timeout_ns (< 0 = no limit). */
int mbe_server_wait(mbe_server* s, uint64_t request_id, int64_t timeout_ns, mbe_result* out);

/* Withdraws a request that is not yet admitted (MBE_OK); one already on the
 * GPU or finished cannot be withdrawn (MBE_ERR_INVALID). */
int mbe_server_cancel(mbe_server* s, uint64_t request_id);

int mbe_server_get_stats(mbe_server* s, mbe_server_stats* out);

/* Diagnosis: a resident request's device counters -- roots claimed, tasks
 * outstanding, roots in all, and its arena block (out[0..3]).
 * MBE_ERR_INVALID if the request is not on the device. */
int mbe_server_debug_request(mbe_server* s, uint64_t request_id, uint64_t out[4]);

/* Biclique lists from the server (no counterpart in the reference, which
 * only counts): every maximal biclique of every request, in original ids and
 * sides, each side ascending, with the request it belongs to.  The return
 * value is ignored. */
typedef int (*mbe_server_emit_fn)(uint64_t request_id, const int32_t* u_ids, int32_t n_u,
                                  const int32_t* v_ids, int32_t n_v, void* user);

/* Turns on emission for every request submitted afterwards; call it before
 * the first submit (MBE_ERR_INVALID after).  Records pass through a
 * host-mapped ring of `ring_words` int32 words (at least max_degree + 2; 0 =
 * 2^22) that the server thread drains while the launch runs, calling `fn`
 * on that thread; a launch whose ring is full waits for it.  A request's
 * result (mbe_server_poll / wait) is reported only after all its bicliques
 * have been passed to `fn`. */
int mbe_server_set_emit(mbe_server* s, int64_t ring_words, mbe_server_emit_fn fn, void* user);

/* Stops the launch (graphs still on the GPU are abandoned) and frees all. */
int mbe_server_destroy(mbe_server* s);

/* ---- measurement (no counterpart in the reference) ------------------------
 * L2 read bandwidth as the SMs see it, for the benchmark's roofline of
 * workloads whose graph fits L2: one launch reads a `bytes` buffer (1-96
 * MiB, device memory it allocates and frees) `passes` (1-1000) times with loads that
 * bypass L1, after a warm-up sweep has brought it into L2; *gbs = bytes read
 * per second / 1e9, timed with CUDA events. */
int mbe_measure_l2_read(int32_t device, int64_t bytes, int32_t passes, double* gbs);

/* ---- synthetic inputs ------------------------------------------------------
 * Seeded Chung-Lu bipartite generator (splitmix64 stream, Vose alias
 * sampling): expected degree of vertex i proportional to (i+1)^(-1/(gamma-1)),
 * capped at max_deg, scaled to ~n_edges; duplicate edges removed, rows sorted,
 * V rows of degree 0 dropped and U ids renumbered densely (so every vertex of
 * either side has an edge).  pair_p_max > 0 caps the probability of any one
 * (u,v) pair at pair_p_max: a draw is kept with probability
 * min(1, -ln(1-pair_p_max) / (w_u w_v / sum w)).  Without the cap, hubs whose
 * weight product exceeds the edge count form a near-complete block whose few
 * missing edges give exponentially many maximal bicliques.  With the cap the
 * edge target is also clamped to pair_p_max * nU * nV.
 * Optional planted blocks: n_blocks disjoint (block_u x block_v) vertex sets,
 * each pair an edge with probability block_p.  Not part of the reference
 * (its inputs are downloaded datasets, preprocess/prepare_dataset.sh). */
typedef struct mbe_gen_spec {
  int64_t nU, nV, n_edges;
  double gamma_u, gamma_v;
  int64_t max_deg_u, max_deg_v;
  uint64_t seed;
  int32_t n_blocks, block_u, block_v, reserved;
  double block_p;
  double pair_p_max; /* 0 = uncapped Chung-Lu */
} mbe_gen_spec;

/* Generate into library-owned arrays (release with mbe_free). *row_off has
 * *nV+1 entries, *col has *nE entries. */
int mbe_gen_chung_lu(const mbe_gen_spec* spec, int32_t** row_off, int32_t** col, int32_t* nV,
                     int32_t* nU, int64_t* nE);

/* The batched-mode size distribution: from `seed`, |U| log-uniform in
 * [50, 5000], |V|/|U| log-uniform in [0.5, 4], average U degree uniform in
 * [3, 30], exponent 2.2 on both sides, expected-degree cap sqrt(edges)
 * (Chung-Lu's condition for edge probabilities below 1), pair probability
 * cap 0.1. */
int mbe_gen_batch_spec(uint64_t seed, mbe_gen_spec* out);

/* Write an .adj file (one line per V row, space-separated ascending U ids). */
int mbe_write_adj(const char* path, const int32_t* row_off, const int32_t* col, int32_t nV);

/* Write the edge-pair .graph form read by the CPU peers (PARMBE, ooMBEA):
 * a first line "<rows> <max id + 1>", then one line "<row> <id>" per entry
 * in row order (replaces preprocess/adj_to_graph.cpp). */
int mbe_write_graph(const char* path, const int32_t* row_off, const int32_t* col, int32_t nV);

/* Parse an .adj file into library-owned host arrays without uploading. */
int mbe_read_adj(const char* path, int32_t** row_off, int32_t** col, int32_t* nV, int32_t* nU,
                 int64_t* nE);

void mbe_free(void* p);

#ifdef __cplusplus
}
#endif

#endif /* GMBE_B200_MBE_H */
