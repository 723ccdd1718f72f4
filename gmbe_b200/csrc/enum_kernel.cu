// The enumeration engine: one persistent kernel, one task per warp.
//
// Semantics follow the reference's GMBE path (the -s 2 kernel):
//   task set-up      IterFinderWithMultipleVertex   src/IterFinderGpu.cu:772-887
//   stack DFS        IterProcess                    src/IterFinderGpu.cu:12-69
//   push / pop       finder_push / finder_pop       src/IterFinderGpu.h:206-303 (PRUNE_EN)
//   task splitting   split test + LargeToTiny       src/IterFinderGpu.cu:835-858, 889-910
//   scheduling       IterFinderKernel_6             src/IterFinderGpu.cu:918-1053
// The data layout and the work per step are this engine's own:
//   * Task set-up counts the two-hop multiset once through a per-warp dense
//     map (no union merges, no binary searches) and lays the candidate set C
//     out as [Q part | P part] instead of sorting it.
//   * Tier 1 (|L| above the bitmap limit) keeps GMBE's per-candidate
//     neighbour counts and level bounds, but walks per-task local adjacency
//     (L position -> C index and C index -> L position) instead of binary
//     searching global rows on every push and pop.
//   * Tier 2 (|L| <= 32*K) re-expresses the same DFS over K-word bitmaps of
//     the current L: a push is an AND, the maximality test a compare, the
//     pro-active pruning test an AND with the removed vertices.
//   * Split tasks go to a bounded MPMC ring; every device wait is bounded and
//     reports a status instead of hanging.
#include <cuda_runtime.h>

#include <cstdio>

#include "enum_common.cuh"
#include "enum_launch.h"

namespace gmbe {

namespace {

constexpr int32_t kFree = 0x7fffffff;     // live at every level (reference 0x7fff)
constexpr int32_t kTouched = 0x3fffffff;  // marked by the pop restore pass (reference 0x3fff)
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned r;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(r));
  return r;
}

__device__ void set_status(EnumCtl* ctl, int32_t code, unsigned long long info) {
  if (atomicCAS(&ctl->status, 0, code) == 0) ctl->err_info = info;
  atomicExch(&ctl->abort, 1);
}

// Whether this warp should leave its task (lane-uniform): the launch is
// aborting, or its time limit has passed (which starts the abort).
template <typename WarpT>
__device__ __forceinline__ bool must_stop(const WarpT& W) {
  int s = 0;
  if (lane_id() == 0) {
    s = *(volatile int32_t*)&W.ctl->abort;
    if (!s && W.deadline != 0) {
      const uint64_t now = globaltimer_ns();
      if (now > W.deadline) {
        set_status(W.ctl, kStDeadline, now - W.deadline);
        s = 1;
      }
    }
  }
  return __shfl_sync(0xffffffffu, s, 0) != 0;
}

// Visits every entry of a list of rows with all 32 lanes busy.  row_of(r, beg,
// len) describes row r; visit(valid, r, pos) is called by every lane (uniform
// control flow), pos indexing the global entry array.
template <typename RowOf, typename Visit>
__device__ __forceinline__ void flat_rows(int nr, RowOf row_of, Visit visit) {
  const int lane = (int)lane_id();
  for (int r0 = 0; r0 < nr; r0 += 32) {
    int r = r0 + lane, beg = 0, len = 0;
    if (r < nr) row_of(r, beg, len);
    int tot;
    int ex = warp_excl_scan(len, &tot);
    for (int e0 = 0; e0 < tot; e0 += 32) {
      int e = e0 + lane;
      int lo = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        int cand = lo + step;
        int exc = __shfl_sync(kFull, ex, cand & 31);
        if (cand < 32 && exc <= e) lo = cand;
      }
      int b = __shfl_sync(kFull, beg, lo);
      int exl = __shfl_sync(kFull, ex, lo);
      bool valid = e < tot;
      visit(valid, r0 + lo, b + (e - exl));
    }
  }
}

struct Warp {
  // Launch constants, read in place from the kernel's parameter space.
  const EnumParams& p;
  const ScratchLayout& sl;
  EnumCtl* ctl;
  Task* q_tasks;
  unsigned long long* q_seq;
  int32_t* slots;        // exported bitmap sub-problems (nslot x slot_words)
  uint32_t* slot_bits;   // slot occupancy
  int nslot;
  int32_t* bigslots;     // large slots (nbig x kBigSlotWords)
  uint32_t* big_bits;
  int nbig;
  int import_cap;        // most candidates any warp of the launch can take in
  int import_l, import_s; // most L vertices / two-hop entries any warp can take in
  int32_t* base;
  const DevGraph* graphs;  // every graph of the launch
  const DevGraph* gp;      // graph of the task being run
  int32_t gid;
  // accumulators (uniform over lanes)
  unsigned long long cnt, hash, nonmax, splits;
  unsigned long long ns_t2, n_t2;  // time inside the bitmap tier, sub-problems run
  unsigned long long pushes;       // pushes so far: counts tier | bitmap tier << 32
  unsigned long long shape;        // last task set up: |C| | (part << 32) | (parts << 48)
  unsigned long long ns_t1;        // time inside the counts tier (bitmap tier excluded)
  uint32_t* seen;                  // this warp's first-touch bitmap in shared memory, or null
  uint64_t deadline;               // %globaltimer after which the launch gives up (0: never)
  uint32_t* gseen;                 // this warp's first-touch bitmap in global memory
  long long dem_t;                 // clock64 of the last export-demand reading (lane 0)
  int dem;                         // that reading

  __device__ int32_t* A(int64_t off) const { return base + off; }
  __device__ uint64_t* A64(int64_t off) const { return reinterpret_cast<uint64_t*>(base + off); }
};

// Adds 1 to counts[i] and tells whether this was i's first touch since the
// counts were last cleared.  With a shared-memory bitmap the first touch is a
// shared atomic and the count a fire-and-forget global one, so the warp does
// not wait for an L2 round trip per entry; without it, the returned old count
// tells.
__device__ __forceinline__ bool count_first(const Warp& W, int32_t* counts, int i) {
  if (W.seen) {
    const uint32_t bit = 1u << (i & 31);
    atomicAdd(&counts[i], 1);
    return (atomicOr(&W.seen[i >> 5], bit) & bit) == 0u;
  }
  return atomicAdd(&counts[i], 1) == 0;
}

// After a counting pass: makes every lane's count increments visible to the
// warp, and clears the bitmap bits of the `n` indices touched (listed in idx).
__device__ __forceinline__ void counts_done(const Warp& W, const int32_t* idx, int n) {
  __threadfence_block();
  __syncwarp();
  if (W.seen) {
    for (int i = (int)lane_id(); i < n; i += 32) W.seen[idx[i] >> 5] = 0u;
    __syncwarp();
  }
}

// Whether a counting pass of `entries` entries over an index space of
// `words` bitmap words collects its first touches from the global bitmap:
// only without the shared-memory bitmap, and when the pass is large enough
// that a scan of the words costs less than an atomic round trip per 32
// entries.
__device__ __forceinline__ bool use_gseen(const Warp& W, long long entries, int words) {
  if (W.p.touch_scan != 0) return W.p.touch_scan > 0;
  return W.seen == nullptr && entries >= (long long)words;
}

// Lists the set bits of bits[0, words) in increasing index order into
// out[0, cap) (indices beyond cap are not written) and clears the words;
// returns the number of set bits.  Every lane takes one word per round, so
// the loads are independent and coalesced.  The bits were set by this warp's
// atomics: the fence before the call makes them visible here.
__device__ int collect_bits(uint32_t* bits, int words, int32_t* out, int cap) {
  const int lane = (int)lane_id();
  int n = 0;
  for (int w0 = 0; w0 < words; w0 += 32) {
    const int w = w0 + lane;
    uint32_t m = w < words ? __ldcg(bits + w) : 0u;
    if (m) bits[w] = 0u;
    int tot;
    int o = n + warp_excl_scan(__popc(m), &tot);
    while (m) {
      if (o < cap) out[o] = (w << 5) + __ffs(m) - 1;
      ++o;
      m &= m - 1;
    }
    n += tot;
  }
  __syncwarp();
  return n;
}

// Emission (opt-in): appends a maximal biclique's L to the launch's record
// buffer as [|L|, graph, internal U ids of L...]; R is N(L).  Two forms:
//  - a buffer (rd null): a record that does not fit entirely is dropped (the
//    reserved word count keeps growing past the buffer, which tells the
//    host); the host zeroes the buffer first and reads it after the launch;
//  - a ring in host-mapped memory (rd = the host's consumed word count):
//    positions grow without bound and index the ring modulo its size; a
//    producer whose record would overrun words the host has not consumed
//    waits for it (bounded by wait_ns: past it the launch fails with a
//    timeout status and the record is dropped).  The host drains the ring
//    while the launch runs and zeroes what it consumed.
// In both, the body and graph words are made visible system-wide before the
// length word, which commits the record (the host waits for a non-zero
// length at the next position).  Kept out of line and given plain
// arguments: inlined at its four call sites, the code grew the
// enumeration's hot loops enough to slow every launch by a quarter.
struct EmitDst {
  int32_t* buf;
  long long cap;                        // words
  const unsigned long long* rd;         // ring: words the host has consumed
  long long wait_ns;                    // ring: longest wait for room
};

__device__ __forceinline__ EmitDst emit_dst(const EnumParams& p) {
  return EmitDst{p.emit, p.emit_cap, p.emit_read, p.idle_ns_limit};
}

// Reserves a record of `count` ids (lane-uniform); -1 if it is dropped.
__device__ long long emit_reserve(EnumCtl* ctl, const EmitDst& d, int count) {
  const unsigned long long need = (unsigned long long)count + 2;
  long long pos = 0;
  if (lane_id() == 0) {
    const unsigned long long at = atomicAdd(&ctl->emit_pos, need);
    if (!d.rd) {
      pos = at + need > (unsigned long long)d.cap ? -1LL : (long long)at;
    } else if (need > (unsigned long long)d.cap) {
      pos = -1;
      set_status(ctl, kStCapacity, ((unsigned long long)6 << 32) | (unsigned)count);
    } else {
      pos = (long long)at;
      const uint64_t t0 = globaltimer_ns();
      while (at + need > *(volatile const unsigned long long*)d.rd + (unsigned long long)d.cap) {
        if (*(volatile int32_t*)&ctl->abort || globaltimer_ns() - t0 > (uint64_t)d.wait_ns) {
          set_status(ctl, kStTimeout, at);
          pos = -1;
          break;
        }
        __nanosleep(1000);
      }
    }
  }
  return __shfl_sync(kFull, pos, 0);
}

__device__ __forceinline__ int32_t& emit_at(const EmitDst& d, long long pos) {
  return d.buf[(unsigned long long)pos % (unsigned long long)d.cap];
}

__device__ __forceinline__ void emit_header(const EmitDst& d, long long pos, int count, int gid) {
  __threadfence_system();
  __syncwarp();
  if (lane_id() == 0) {
    emit_at(d, pos + 1) = gid;
    __threadfence_system();
    emit_at(d, pos) = count;
  }
  __syncwarp();
}

// L = ids[idx[i]] (or ids[i] when idx is null) for i < n.
__device__ __noinline__ void emit_list(EnumCtl* ctl, EmitDst d, int gid, int n,
                                       const int32_t* ids, const int32_t* idx) {
  const long long pos = emit_reserve(ctl, d, n);
  if (pos < 0) return;
  for (int i = (int)lane_id(); i < n; i += 32) emit_at(d, pos + 2 + i) = idx ? ids[idx[i]] : ids[i];
  emit_header(d, pos, n, gid);
}

// L = ids[l] for the l < nscan with llevel[l] == level, count of them.
__device__ __noinline__ void emit_level(EnumCtl* ctl, EmitDst d, int gid, int count, int nscan,
                                        const int32_t* llevel, int level, const int32_t* ids) {
  const long long pos = emit_reserve(ctl, d, count);
  if (pos < 0) return;
  int out = 0;
  for (int b0 = 0; b0 < nscan; b0 += 32) {
    const int l = b0 + (int)lane_id();
    const bool s = l < nscan && llevel[l] == level;
    const unsigned bal = __ballot_sync(kFull, s);
    if (s) emit_at(d, pos + 2 + out + __popc(bal & lanemask_lt())) = ids[l];
    out += __popc(bal);
  }
  emit_header(d, pos, count, gid);
}

// L = lid[b] for the set bits b of the K-word mask (m0..m3), count of them.
__device__ __noinline__ void emit_mask(EnumCtl* ctl, EmitDst d, int gid, int count, int K,
                                       uint32_t m0, uint32_t m1, uint32_t m2, uint32_t m3,
                                       const int32_t* lid) {
  const long long pos = emit_reserve(ctl, d, count);
  if (pos < 0) return;
  const int lane = (int)lane_id();
  int out = 0;
  for (int w = 0; w < K; ++w) {
    const uint32_t m = w == 0 ? m0 : (w == 1 ? m1 : (w == 2 ? m2 : m3));
    const bool s = (m >> lane) & 1u;
    if (s) emit_at(d, pos + 2 + out + __popc(m & lanemask_lt())) = lid[w * 32 + lane];
    out += __popc(m);
  }
  emit_header(d, pos, count, gid);
}

// Serving block of graph `gid` (a block index into the arena, which the
// launch receives in place of the descriptor array).
__device__ __forceinline__ ServeGraph* serve_graph(const Warp& W, int32_t gid) {
  char* arena = const_cast<char*>(reinterpret_cast<const char*>(W.graphs));
  return reinterpret_cast<ServeGraph*>(arena + ((size_t)(uint32_t)gid << kServeBlockShift));
}

// Descriptor of graph `gid` of this launch.
__device__ __forceinline__ const DevGraph* graph_at(const Warp& W, int32_t gid) {
  return W.p.server ? &serve_graph(W, gid)->g : W.graphs + gid;
}

// Most parts a root is split into.
constexpr int kMaxParts = 1024;

// Bucket of candidate w among `parts` (Knuth's multiplicative hash, scaled):
// spreads consecutive ids, hence the work, evenly over the parts.
__device__ __forceinline__ int part_of(int w, int parts) {
  return (int)(((unsigned long long)((uint32_t)w * 2654435761u) * (unsigned)parts) >> 32);
}

// Children of the current graph about to be queued (serving: a graph
// completes when its roots and every queued child have finished).
__device__ __forceinline__ void graph_spawned(const Warp& W, unsigned long long n) {
  if (W.p.server) atomicAdd(&serve_graph(W, W.gid)->pending, n);
}

// ---------------------------------------------------------------------------
// Bitmap sub-problems.
//
// A sub-problem is an L of at most 128 vertices (K = 1, 2 or 4 words) and a
// list of candidate records of rec_stride(K) words: word 0 = (index << 8) | bound,
// words 1..K = the candidate's neighbourhood inside L.  index is the
// candidate's position in the sub-problem, whose order is [Q | P]; bound is
// GMBE's level bound in 8 bits (kB8Free = live at every level; levels stay
// at or below 129).  subkey[index] is the candidate's hash key, lkey[b] that
// of L bit b.
constexpr uint32_t kB8Free = 255;
// Words per record: K + 1, except that K = 2 records are padded to 4 words so
// that one 16-byte access reads or writes a record (one-word records are one
// 8-byte access).  Lists start at 32-byte aligned scratch slices or slots and
// follow one another in whole records, so K = 1 and K = 2 lists stay 8- and
// 16-byte aligned.
__host__ __device__ constexpr int rec_stride(int K) { return K == 2 ? 4 : K + 1; }

struct T2Src {
  uint32_t* rec;           // nsub records, writable (their bounds change)
  const uint64_t* subkey;
  const uint64_t* lkey;
  const int32_t* lid;      // internal U id of each L bit (emission only)
  uint32_t L0[4];          // the sub-problem's L
  int nsub, nq;            // records [0, nq) are Q, [nq, nsub) P
  int nend;                // the first level pushes records [nq, nend) only
  uint64_t sR0;            // R of the sub-problem's root biclique
  uint32_t nR0;
};

// Slot layout (int32 words): header, lkey (128 x uint64), records, subkey.
constexpr int kSlotWords = 32768;
constexpr int kSlotHdr = 16;
constexpr int kSlotLkey = kSlotHdr;
constexpr int kSlotLid = kSlotLkey + 2 * 32 * 4;  // 128 int32: the L bits' vertex ids
constexpr int kSlotRec = kSlotLid + 32 * 4;
__host__ __device__ constexpr int slot_cap(int K) {
  return ((kSlotWords - kSlotRec - 2) / (rec_stride(K) + 2)) & ~31;
}
__host__ __device__ constexpr int big_slot_cap(int K) {
  return ((kBigSlotWords - kSlotRec - 2) / (rec_stride(K) + 2)) & ~31;
}
static_assert(slot_cap(1) == kSlotMaxRecords && slot_cap(1) >= slot_cap(2) &&
                  slot_cap(2) >= slot_cap(4) && kSlotWords == kSlotWordsHost,
              "host view of the slot size");
// header words: 0 K, 1 nsub, 2 nq, 3 graph, 4..7 L0, 8..9 sR0, 10 nR0
__device__ __forceinline__ uint64_t* slot_subkey(int32_t* sp, int K, int nsub) {
  return reinterpret_cast<uint64_t*>(sp + kSlotRec + ((nsub * rec_stride(K) + 1) & ~1));
}

// Claims a free slot of an occupancy bitmap of n slots (lane 0); -1 if none.
__device__ int bits_alloc(uint32_t* bits, int n) {
  const int nw = n >> 5;
  if (nw == 0) return -1;
  int start = (int)(((blockIdx.x * 32u + (threadIdx.x >> 5)) * 2654435761u) % (unsigned)nw);
  for (int t = 0; t < nw; ++t) {
    int wi = (start + t) % nw;
    unsigned cur = *(volatile unsigned*)&bits[wi];
    while (cur != 0xffffffffu) {
      int b = __ffs(~cur) - 1;
      unsigned old = atomicOr(&bits[wi], 1u << b);
      if (!(old & (1u << b))) return wi * 32 + b;
      cur = old | (1u << b);
    }
  }
  return -1;
}

// A regular slot (lane 0); -1 if none.
__device__ int slot_alloc(Warp& W) { return bits_alloc(W.slot_bits, W.nslot); }

// A slot for a sub-problem of nsub candidates with K-word masks (lane 0): a
// regular one when it fits, else a large one if some warp of every tier can
// take it in; -1 if none.
__device__ __forceinline__ bool regular_fits(const Warp& W, int nsub, int K) {
  return nsub <= slot_cap(K) && (W.p.slot_records <= 0 || nsub <= W.p.slot_records);
}

__device__ int slot_alloc_for(Warp& W, int nsub, int K) {
  if (regular_fits(W, nsub, K)) return slot_alloc(W);
  if (nsub > big_slot_cap(K) || nsub > W.import_cap) return -1;
  const int b = bits_alloc(W.big_bits, W.nbig);
  return b < 0 ? -1 : W.nslot + b;
}

// Whether a child of nsub candidates can be exported at all.
__device__ __forceinline__ bool slot_fits(const Warp& W, int nsub, int K) {
  return regular_fits(W, nsub, K) ||
         (W.nbig > 0 && nsub <= big_slot_cap(K) && nsub <= W.import_cap);
}

__device__ __forceinline__ int32_t* slot_ptr(const Warp& W, int s) {
  return s < W.nslot ? W.slots + (size_t)s * kSlotWords
                     : W.bigslots + (size_t)(s - W.nslot) * kBigSlotWords;
}

__device__ void slot_free(Warp& W, int s) {
  if (s < W.nslot) atomicAnd(&W.slot_bits[s >> 5], ~(1u << (s & 31)));
  else {
    const int b = s - W.nslot;
    atomicAnd(&W.big_bits[b >> 5], ~(1u << (b & 31)));
  }
}

__device__ bool queue_push_one(Warp& W, const Task& t);

// Demand for exported work (lane-uniform): 0 none, 1 idle warps outnumber
// queued work, 2 more than an eighth of all warps are idle as well.
// The counters are global loads the warp would wait for on every sizable
// child, so a reading is reused for kDemandCycles SM clocks (about 2 us):
// demand moves with warps going idle, far more slowly than children come.
constexpr long long kDemandCycles = 4096;
__device__ int export_demand(Warp& W) {
  int want = 0;
  if (lane_id() == 0) {
    const long long now = clock64();
    if (now - W.dem_t < kDemandCycles) {
      want = W.dem;
    } else {
      EnumCtl* c = W.ctl;
      int idle = *(volatile int32_t*)&c->idle_warps;
      unsigned long long queued = *(volatile unsigned long long*)&c->q_tail -
                                  *(volatile unsigned long long*)&c->q_head;
      if (idle > 0 && (unsigned long long)idle > queued) {
        const int warps = (int)(gridDim.x * (blockDim.x >> 5));
        want = idle > (warps >> 3) ? 2 : 1;
      }
      W.dem = want;
      W.dem_t = now;
    }
  }
  return __shfl_sync(0xffffffffu, want, 0);
}

// GMBE's split test on a child: (|P| > h or |L| > h) and |P| * |L| > s.
__device__ __forceinline__ bool big_enough(const Warp& W, int nP, int nL) {
  return (nP > W.gp->bound_height || nL > W.gp->bound_height) &&
         (long long)nP * nL > (long long)W.gp->bound_size;
}

// Whether to hand a child (nP P-candidates, |L| = nL) to another warp.  A
// child that passes GMBE's split test goes whenever warps wait for work.
// When many warps wait, smaller children go too: the size test misjudges
// dense graphs, where a few dozen candidates can hold millions of
// bicliques.  The floor (share_min_work) keeps the tiniest children, whose
// copy would cost the exporting warp more than running them, at home.
// `eager`: a child that passes the split test goes even when no warp waits
// (the counts tier's parents are the heaviest tasks of a launch and are
// claimed first; their children, queued ahead of new roots, keep every warp
// busy instead of lengthening the parent).
__device__ bool should_export(Warp& W, int nP, int nL, bool eager = false) {
  if (nP < 2 || nL < 2) return false;
  const bool big = big_enough(W, nP, nL);
  const bool sizable = (long long)nP * nL >= W.p.share_min_work;
  if (!big && !sizable) return false;  // goes at no demand: skip reading it
  if (eager && big) return true;
  const int d = export_demand(W);
  return (d == 2 && (big || sizable)) || (d == 1 && big);
}

// Enqueues a filled slot as a task; false if the ring is full.
// kind 0: a bitmap sub-problem; kind 1: a counts-tier child (vertex lists).
__device__ bool slot_publish(Warp& W, int slot, int kind = 0) {
  __syncwarp();
  __threadfence();
  Task t;
  t.v[0] = -2 - slot;
  t.v[1] = kind ? 1 : -1;
  t.v[2] = t.v[3] = -1;
  t.graph = t.part = t.parts = t.pad = 0;
  return queue_push_one(W, t);
}

__device__ void slot_header(int32_t* sp, int K, int nsub, int nq, const uint32_t* L0, uint64_t sR,
                            uint64_t nR, int gid) {
  sp[0] = K;
  sp[1] = nsub;
  sp[2] = nq;
  sp[3] = gid;
  for (int w = 0; w < 4; ++w) sp[4 + w] = w < K ? (int32_t)L0[w] : 0;
  *reinterpret_cast<uint64_t*>(sp + 8) = sR;
  sp[10] = (int32_t)nR;
}

// Exports the child of a push of a bitmap sub-problem (its records
// `child`, in order, the first nbefore of them Q) to an idle warp.
template <int K>
__device__ bool t2_try_export(Warp& W, const T2Src& src, const uint32_t* child, int nchild,
                              int nbefore, const uint32_t* Ln, int kn, uint64_t sR, uint64_t nR) {
  if (!slot_fits(W, nchild, K) || !should_export(W, nchild - nbefore, kn))
    return false;
  const int lane = (int)lane_id();
  int slot = lane == 0 ? slot_alloc_for(W, nchild, K) : 0;
  slot = __shfl_sync(0xffffffffu, slot, 0);
  if (slot < 0) return false;
  constexpr int RS = rec_stride(K);
  int32_t* sp = slot_ptr(W, slot);
  uint32_t* rec = reinterpret_cast<uint32_t*>(sp + kSlotRec);
  uint64_t* key = slot_subkey(sp, K, nchild);
  uint64_t* lk = reinterpret_cast<uint64_t*>(sp + kSlotLkey);
  for (int q = lane; q < nchild; q += 32) {
    const uint32_t* c = child + (size_t)q * RS;
    rec[(size_t)q * RS] = ((uint32_t)q << 8) | kB8Free;
#pragma unroll
    for (int w = 0; w < K; ++w) rec[(size_t)q * RS + 1 + w] = c[1 + w];
    key[q] = src.subkey[c[0] >> 8];
  }
  for (int b = lane; b < 32 * K; b += 32) lk[b] = src.lkey[b];
  if (W.p.emit) {  // L ids are needed for emission only
    int32_t* li = sp + kSlotLid;
    for (int b = lane; b < 32 * K; b += 32) li[b] = src.lid[b];
  }
  if (lane == 0) slot_header(sp, K, nchild, nbefore, Ln, sR, nR, W.gid);
  if (slot_publish(W, slot)) return true;
  if (lane == 0) slot_free(W, slot);
  __syncwarp();
  return false;
}

// ---------------------------------------------------------------------------
// Tier 2: the DFS of IterProcess / finder_push / finder_pop on a bitmap
// sub-problem.  Every level owns a contiguous record list: the candidates
// that still meet the level's L and are neither absorbed nor retired
// (MBEA's shrinking P and Q), copied with their masks so each pass is a
// unit-stride sweep.  Level bounds live in the records: a deeper level only
// changes its own copies, which is equivalent to GMBE's shared bound array
// because a pop at a level re-derives every bound >= that level.  A child
// list that does not fit the arena shares its parent's records (GMBE's
// shared-array semantics for that pair of levels).  R of the push that
// opened a level is carried on the stack: absorbed candidates leave the
// lists but stay in every R below.
//
// finder_pop is not a pass of its own: a pop at a level is only remembered
// (the candidate and the L vertices it leaves, `rem`), and its bound rule is
// applied record by record by the next pass over the level, the scan for the
// next candidate and that candidate's push, which write each header once.
// A level that ends with a pop pending drops it: its records are discarded,
// or (a list shared with the parent) every bound the pop would set is one
// the parent's own pop re-derives.
template <int K>
__device__ void tier2_run(Warp& W, const T2Src& src) {
  constexpr int RS = rec_stride(K);
  const int lane = (int)lane_id();
  const uint64_t* subkey = src.subkey;
  const uint64_t* lkey = src.lkey;
  uint32_t* arena = reinterpret_cast<uint32_t*>(W.A(W.sl.act));
  const int actcap = W.sl.act_cap;
  uint64_t* lrec = W.A64(W.sl.t2_rec);   // record list of each level
  int32_t* ln = W.A(W.sl.t2_n);          // its length
  int32_t* lcur = W.A(W.sl.t2_cur);      // scan position in it
  int32_t* ltop = W.A(W.sl.t2_top);      // first free arena word above it
  uint32_t* lmask = reinterpret_cast<uint32_t*>(W.A(W.sl.lmask));
  uint64_t* rsum = W.A64(W.sl.r_sum);
  uint32_t* rcnt = reinterpret_cast<uint32_t*>(W.A(W.sl.r_cnt));
  const bool emitting = W.p.emit != nullptr;
  const bool prune = W.p.prune != 0;

  for (int q = lane; q < src.nsub; q += 32) {
    uint32_t h = src.rec[(size_t)q * RS];
    src.rec[(size_t)q * RS] = (h & ~0xffu) | kB8Free;
  }
  if (lane == 0) {
    lrec[0] = reinterpret_cast<uint64_t>(src.rec);
    ln[0] = src.nsub;
    lcur[0] = src.nq;
    ltop[0] = 0;
    rsum[0] = src.sR0;
    rcnt[0] = src.nR0;
  }
  if (lane < K) {
    uint32_t v = 0;
#pragma unroll
    for (int w = 0; w < K; ++w)
      if (w == lane) v = src.L0[w];
    lmask[lane] = v;
  }
  __syncwarp();
  int level = 1;
  unsigned steps = 0;
  // The pending pop at `level`: its candidate (-1: none) and the L vertices
  // of the level it does not meet.
  int pcp = -1;
  uint32_t prem[K];
#pragma unroll
  for (int w = 0; w < K; ++w) prem[w] = 0u;
  // A record's bound after the pending pop (finder_pop: a bound >= level is
  // re-derived, FREE if the record meets rem or is the popped one, else
  // level - 1; without pruning always FREE).
  auto popped = [&](int q, uint32_t b, const uint32_t* m) -> uint32_t {
    if (pcp < 0 || (int)b < level) return b;
    if (!prune || q == pcp) return kB8Free;
    uint32_t any = 0;
#pragma unroll
    for (int w = 0; w < K; ++w) any |= m[w] & prem[w];
    return any ? kB8Free : (uint32_t)(level - 1);
  };
  while (level != 0) {
    if ((++steps & 4095u) == 0u && must_stop(W)) return;
    uint32_t* R = reinterpret_cast<uint32_t*>(lrec[level - 1]);
    const int n = ln[level - 1];
    uint32_t Lm[K];
#pragma unroll
    for (int w = 0; w < K; ++w) Lm[w] = lmask[(level - 1) * K + w];
    int cp = -1;
    const int e = level == 1 ? src.nend : n;  // the first level may push a part only
    for (int b0 = lcur[level - 1]; b0 < e; b0 += 32) {
      int q = b0 + lane;
      bool ok = false;
      if (q < e) {
        uint32_t h, m[K];
        if constexpr (K == 1) {
          // One 8-byte load per record (lists start 8-byte aligned, records
          // are two words): half the load instructions and L1 wavefronts.
          const uint2 hm = reinterpret_cast<const uint2*>(R)[q];
          h = hm.x;
          m[0] = hm.y;
        } else if constexpr (K == 2) {
          const uint4 hm = reinterpret_cast<const uint4*>(R)[q];  // padded to 4 words
          h = hm.x;
          m[0] = hm.y;
          m[1] = hm.z;
        } else {
          const uint32_t* r = R + (size_t)q * RS;
          h = r[0];
#pragma unroll
          for (int w = 0; w < K; ++w) m[w] = r[1 + w];
        }
        if ((int)popped(q, h & 0xffu, m) > level - 1) {
          uint32_t any = 0;
#pragma unroll
          for (int w = 0; w < K; ++w) any |= m[w] & Lm[w];
          ok = any != 0;
        }
      }
      unsigned bal = __ballot_sync(kFull, ok);
      if (bal) {
        cp = b0 + __ffs(bal) - 1;
        break;
      }
    }
    if (cp >= 0) {
      // ---- push (finder_push) ----
      W.pushes += 1ULL << 32;
      uint32_t Ln[K];
      int kn = 0;
#pragma unroll
      for (int w = 0; w < K; ++w) {
        Ln[w] = Lm[w] & R[(size_t)cp * RS + 1 + w];
        kn += __popc(Ln[w]);
      }
      const int ctop = ltop[level - 1];
      const bool fits = ctop + n * RS <= actcap;
      uint32_t* child = arena + ctop;
      bool ism = true;
      uint64_t sR = 0;
      unsigned long long nR = 0;
      int nchild = 0, nbefore = 0;
      // The pass is bound by load latency: each lane loads U records before
      // any of them is used, so U loads per lane are in flight at once.
      constexpr int U = K <= 2 ? 4 : 2;
      for (int b0 = 0; b0 < n; b0 += 32 * U) {
        uint32_t hu[U], mu[U][K];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int q = b0 + u * 32 + lane;
          hu[u] = 0u;
#pragma unroll
          for (int w = 0; w < K; ++w) mu[u][w] = 0u;
          if (q < n) {
            if constexpr (K == 1) {
              const uint2 hm = reinterpret_cast<const uint2*>(R)[q];
              hu[u] = hm.x;
              mu[u][0] = hm.y;
            } else if constexpr (K == 2) {
              const uint4 hm = reinterpret_cast<const uint4*>(R)[q];
              hu[u] = hm.x;
              mu[u][0] = hm.y;
              mu[u][1] = hm.z;
            } else {
              const uint32_t* r = R + (size_t)q * RS;
              hu[u] = r[0];
#pragma unroll
              for (int w = 0; w < K; ++w) mu[u][w] = r[1 + w];
            }
          }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int q = b0 + u * 32 + lane;
          const uint32_t h = hu[u];
          bool keep = false;
          if (q < n) {
            bool cover = true, meet = false;
#pragma unroll
            for (int w = 0; w < K; ++w) {
              uint32_t x = mu[u][w] & Ln[w];
              cover &= x == Ln[w];
              meet |= x != 0;
            }
            const uint32_t b0h = h & 0xffu;
            const int b = (int)popped(q, b0h, mu[u]);
            uint32_t nb = (uint32_t)b;
            if (cover) {
              sR += subkey[h >> 8];
              ++nR;
              if (q < cp && b >= level) ism = false;
              else if (b > level) nb = (uint32_t)level;
            } else {
              keep = meet && b > level;
            }
            if (nb != b0h) R[(size_t)q * RS] = (h & ~0xffu) | nb;
          }
          unsigned bal = __ballot_sync(kFull, keep);
          if (fits && keep) {
            const int ci = nchild + __popc(bal & lanemask_lt());
            if constexpr (K == 1) {
              reinterpret_cast<uint2*>(child)[ci] = make_uint2((h & ~0xffu) | kB8Free, mu[u][0]);
            } else if constexpr (K == 2) {
              reinterpret_cast<uint4*>(child)[ci] =
                  make_uint4((h & ~0xffu) | kB8Free, mu[u][0], mu[u][1], 0u);
            } else {
              uint32_t* c = child + (size_t)ci * RS;
              c[0] = (h & ~0xffu) | kB8Free;
#pragma unroll
              for (int w = 0; w < K; ++w) c[1 + w] = mu[u][w];
            }
          }
          nchild += __popc(bal);
          nbefore += __popc(__ballot_sync(kFull, keep && q < cp));
        }
      }
      pcp = -1;  // applied by this pass
      ism = __all_sync(kFull, ism);
      sR = warp_sum(sR) + rsum[level - 1];
      nR = warp_sum(nR) + rcnt[level - 1];
      if (ism) {
        uint64_t sL = 0;
#pragma unroll
        for (int w = 0; w < K; ++w)
          if ((Ln[w] >> lane) & 1u) sL += lkey[w * 32 + lane];
        sL = warp_sum(sL);
        W.cnt += 1;
        W.hash += biclique_hash(*W.gp, sL, (uint64_t)kn, sR, nR);
        if (emitting)
          emit_mask(W.ctl, emit_dst(W.p), W.gid, kn, K, Ln[0], K > 1 ? Ln[1 % K] : 0u,
                    K > 2 ? Ln[2 % K] : 0u, K > 3 ? Ln[3 % K] : 0u, src.lid);
      } else {
        W.nonmax += 1;
      }
      __syncwarp();
      // A big enough child goes to an idle warp instead, at any depth, so a
      // subtree that started inline can still be shared once warps run out of
      // work (the state after the pop below does not depend on the child).
      bool exported = false;
      if (ism && kn > 1 && nchild > 0 && fits)
        exported = t2_try_export<K>(W, src, child, nchild, nbefore, Ln, kn, sR, nR);
      if (ism && kn > 1 && nchild > 0 && !exported) {
        if (lane == 0) {
          lcur[level - 1] = cp;
          rsum[level] = sR;
          rcnt[level] = (uint32_t)nR;
          if (fits) {
            lrec[level] = reinterpret_cast<uint64_t>(child);
            ln[level] = nchild;
            lcur[level] = nbefore;  // the child takes candidates after cp
            ltop[level] = ctop + nchild * RS;
          } else {
            lrec[level] = lrec[level - 1];
            ln[level] = n;
            lcur[level] = cp + 1;
            ltop[level] = ctop;
          }
        }
        if (lane < K) {
          uint32_t v = 0;
#pragma unroll
          for (int w = 0; w < K; ++w)
            if (w == lane) v = Ln[w];
          lmask[level * K + lane] = v;
        }
        __syncwarp();
        ++level;
        continue;
      }
      if (lane == 0) lcur[level - 1] = cp + 1;
    } else {
      --level;  // the ended level's pending pop (if any) is dropped
      if (level == 0) break;
      cp = lcur[level - 1];
      __syncwarp();
      if (lane == 0) lcur[level - 1] = cp + 1;
    }
    // ---- pop (finder_pop) of the candidate at position cp of `level`:
    // remembered, applied by the next pass over the level ----
    {
      const uint32_t* R2 = reinterpret_cast<const uint32_t*>(lrec[level - 1]);
      pcp = cp;
#pragma unroll
      for (int w = 0; w < K; ++w)
        prem[w] = lmask[(level - 1) * K + w] & ~R2[(size_t)cp * RS + 1 + w];
    }
    __syncwarp();
  }
}

__device__ void tier2_dispatch(Warp& W, const T2Src& src, int words) {
  uint64_t t0 = globaltimer_ns();
  if (words <= 1) tier2_run<1>(W, src);
  else if (words <= 2) tier2_run<2>(W, src);
  else tier2_run<4>(W, src);
  W.ns_t2 += globaltimer_ns() - t0;
  W.n_t2 += 1;
}

__device__ __forceinline__ int words_k(int n) {
  int w = (n + 31) >> 5;
  return w <= 1 ? 1 : (w <= 2 ? 2 : 4);
}

__device__ __forceinline__ void full_mask(uint32_t* L0, int n) {
#pragma unroll
  for (int w = 0; w < 4; ++w) {
    int bits = n - 32 * w;
    L0[w] = bits >= 32 ? 0xffffffffu : (bits <= 0 ? 0u : ((1u << bits) - 1u));
  }
}

// Sub-problem built in the warp's own scratch over n L vertices (all bits).
__device__ void tier2(Warp& W, int n, int nsub, int nq, int nend, uint64_t sR0, uint64_t nR0) {
  T2Src src;
  src.rec = reinterpret_cast<uint32_t*>(W.A(W.sl.masks));
  src.subkey = W.A64(W.sl.sub_v);
  src.lkey = W.A64(W.sl.lkey);
  src.lid = W.A(W.sl.lid);
  full_mask(src.L0, n);
  src.nsub = nsub;
  src.nq = nq;
  src.nend = nend;
  src.sR0 = sR0;
  src.nR0 = (uint32_t)nR0;
  tier2_dispatch(W, src, words_k(n));
}

// Runs an exported sub-problem and releases its slot.  The slot was written
// by another warp, possibly on another SM, and this SM may hold lines of it
// from an older owner in its (non-coherent) L1: the header is read with
// volatile loads and the body is copied through L2 (ld.global.cg) into this
// warp's own scratch, where the sub-problem then runs.  The slot is freed as
// soon as it is copied; nothing here writes it, so no store can land on the
// records of its next owner.
__device__ void tier2_from_slot(Warp& W, int slot) {
  const int lane = (int)lane_id();
  int32_t* sp = slot_ptr(W, slot);
  volatile const int32_t* vh = sp;
  const int K = vh[0];
  const int nsub = vh[1];
  const int nq = vh[2];
  const int32_t gid = vh[3];
  T2Src src;
  for (int w = 0; w < 4; ++w) src.L0[w] = (uint32_t)vh[4 + w];
  src.sR0 = (uint64_t)(uint32_t)vh[8] | ((uint64_t)(uint32_t)vh[9] << 32);
  src.nR0 = (uint32_t)vh[10];
  const int RS = rec_stride(K);
  uint32_t* rec = reinterpret_cast<uint32_t*>(W.A(W.sl.masks));
  uint64_t* subkey = W.A64(W.sl.sub_v);
  uint64_t* lkey = W.A64(W.sl.lkey);
  const unsigned* srec = reinterpret_cast<const unsigned*>(sp + kSlotRec);
  const unsigned long long* skey =
      reinterpret_cast<const unsigned long long*>(slot_subkey(sp, K, nsub));
  const unsigned long long* slk = reinterpret_cast<const unsigned long long*>(sp + kSlotLkey);
  const int nw = nsub * RS;
  for (int i = lane; i < nw; i += 32) rec[i] = __ldcg(srec + i);
  for (int i = lane; i < nsub; i += 32) subkey[i] = __ldcg(skey + i);
  int32_t* lid = W.A(W.sl.lid);
  const unsigned* sli = reinterpret_cast<const unsigned*>(sp + kSlotLid);
  for (int i = lane; i < 32 * K; i += 32) lkey[i] = __ldcg(slk + i);
  if (W.p.emit)
    for (int i = lane; i < 32 * K; i += 32) lid[i] = (int32_t)__ldcg(sli + i);
  __syncwarp();
  if (lane == 0) slot_free(W, slot);
  __syncwarp();
  W.gid = gid;
  W.gp = graph_at(W, gid);
  src.rec = rec;
  src.subkey = subkey;
  src.lkey = lkey;
  src.lid = lid;
  src.nsub = nsub;
  src.nq = nq;
  src.nend = nsub;
  tier2_dispatch(W, src, K);
}

// Zeroes nsub records of K mask words, each with its index and a free bound.
__device__ void init_records(uint32_t* rec, int K, int nsub) {
  const int lane = (int)lane_id();
  const int RS = rec_stride(K);
  for (int q = lane; q < nsub; q += 32) {
    rec[(size_t)q * RS] = ((uint32_t)q << 8) | kB8Free;
    for (int w = 0; w < K; ++w) rec[(size_t)q * RS + 1 + w] = 0u;
  }
  __syncwarp();
}

// ---------------------------------------------------------------------------
// Tier 1: GMBE counts + level bounds over the task's C, local adjacency.
struct T1 {
  const int32_t* L;   // L vertices (internal U ids)
  int nL, nC, nq;
  int nend;  // the first level pushes positions [nq, nend) only
  uint64_t sRtask, nRtask;
};

// Selects L positions with Llevel == lvl, calling fn(pos) over rows of aadj.
template <typename Fn>
__device__ __forceinline__ void t1_rows_at_level(Warp& W, const T1& t, int lvl, Fn fn) {
  const int32_t* llevel = W.A(W.sl.llevel);
  const int32_t* aoff = W.A(W.sl.aoff);
  const int lane = (int)lane_id();
  // Compact the selected rows of each 32-chunk, then walk them flat.
  for (int c0 = 0; c0 < t.nL; c0 += 32) {
    int l = c0 + lane;
    bool sel = l < t.nL && llevel[l] == lvl;
    unsigned bal = __ballot_sync(kFull, sel);
    int nsel = __popc(bal);
    if (nsel == 0) continue;
    // Lane j takes the j-th selected row of the chunk (nsel <= 32, so the
    // row index flat_rows passes to row_of is this lane's own id).
    int myrow = -1;
    {
      unsigned m = bal;
      for (int k = 0; k < lane && m; ++k) m &= m - 1;
      if (lane < nsel) myrow = c0 + __ffs(m) - 1;
    }
    flat_rows(
        nsel,
        [&](int, int& beg, int& len) {
          beg = aoff[myrow];
          len = aoff[myrow + 1] - beg;
        },
        fn);
  }
}

// Selects the L positions of candidate x's row (cadj) with llevel == lvl,
// calling fn(pos) over their rows of aadj: the rows a push of x keeps, walked
// without a pass over all of L.
template <typename Fn>
__device__ __forceinline__ void t1_rows_of(Warp& W, int x, int lvl, Fn fn) {
  const int32_t* llevel = W.A(W.sl.llevel);
  const int32_t* aoff = W.A(W.sl.aoff);
  const int32_t* coff = W.A(W.sl.coff);
  const int32_t* cadj = W.A(W.sl.cadj);
  const int lane = (int)lane_id();
  const int rb = coff[x], re = coff[x + 1];
  for (int c0 = rb; c0 < re; c0 += 32) {
    const int j = c0 + lane;
    const int l = j < re ? cadj[j] : 0;
    const bool sel = j < re && llevel[l] == lvl;
    const unsigned bal = __ballot_sync(kFull, sel);
    const int nsel = __popc(bal);
    if (nsel == 0) continue;
    int myrow = -1;
    {
      unsigned m = bal;
      for (int k = 0; k < lane && m; ++k) m &= m - 1;
      if (lane < nsel) myrow = __shfl_sync(kFull, l, __ffs(m) - 1);
      else __shfl_sync(kFull, l, 0);
    }
    flat_rows(
        nsel,
        [&](int, int& beg, int& len) {
          beg = aoff[myrow];
          len = aoff[myrow + 1] - beg;
        },
        fn);
  }
}

// finder_pop (src/IterFinderGpu.h:266-303) of candidate x at `level`, walking
// only the rows of the level above it: the removed rows (llevel == level-1)
// restore their counts and mark the candidates they meet, and the kept rows
// (llevel == level, the rows of x) decide the pruning.  A pass over every
// candidate is not needed: a candidate adjacent to neither kept nor removed
// rows has count 0 at this level and every level below it, so no push, scan,
// maximality test or later pop at or below this level reads its bound, and
// the pop one level up treats every bound >= level-1 alike.
__device__ void t1_pop(Warp& W, const T1& t, int x, int level) {
  int32_t* llevel = W.A(W.sl.llevel);
  int32_t* ncnt = W.A(W.sl.ncnt);
  int32_t* bound = W.A(W.sl.bound);
  const int32_t* aadj = W.A(W.sl.aadj);
  const int32_t* coff = W.A(W.sl.coff);
  const int32_t* cadj = W.A(W.sl.cadj);
  const int lane = (int)lane_id();
  const bool prune = W.p.prune != 0;
  // restore counts over L_parent \ L_child and mark touched candidates
  t1_rows_at_level(W, t, level - 1, [&](bool valid, int, int pos) {
    if (!valid) return;
    int p = aadj[pos];
    if (p < 0) return;
    atomicAdd(&ncnt[p], 1);
    if (bound[p] >= level) bound[p] = kTouched;
  });
  __syncwarp();
  if (prune) {
    // Candidates of the kept rows that no removed row met are retired at this
    // level (a candidate in several kept rows is visited several times: the
    // write is the same each time, and touched ones are left for the pass
    // below).
    t1_rows_of(W, x, level, [&](bool valid, int, int pos) {
      if (!valid) return;
      const int p = aadj[pos];
      if (p < 0 || p == x) return;
      const int b = bound[p];
      if (b >= level && b != kTouched) bound[p] = level - 1;
    });
    __syncwarp();
    // touched candidates -> free
    t1_rows_at_level(W, t, level - 1, [&](bool valid, int, int pos) {
      if (!valid) return;
      const int p = aadj[pos];
      if (p >= 0 && bound[p] == kTouched) bound[p] = kFree;
    });
    __syncwarp();
  }
  if (lane == 0) bound[x] = kFree;
  __syncwarp();
  // the kept rows go back to the level above (deeper levels are popped already)
  for (int j = coff[x] + lane; j < coff[x + 1]; j += 32) {
    const int l = cadj[j];
    if (llevel[l] == level) llevel[l] = level - 1;
  }
  __syncwarp();
}

// Hands the child sub-problem of a maximal push (x at `level`, |L_new| = kept)
// to tier 2.  Candidates: C entries live below this level with
// 0 < count < kept; Q = those before x.
__device__ void t1_handoff(Warp& W, const T1& t, int x, int level, int kept, uint64_t sR,
                           uint64_t nR) {
  const int lane = (int)lane_id();
  const int32_t* llevel = W.A(W.sl.llevel);
  const int32_t* ncnt = W.A(W.sl.ncnt);
  const int32_t* bound = W.A(W.sl.bound);
  const int32_t* cv = W.A(W.sl.cv);
  const uint64_t* ckey = W.A64(W.sl.ckey);
  int32_t* sidx = W.A(W.sl.sidx);
  int32_t* lp = W.A(W.sl.lp);
  uint64_t* lkey = W.A64(W.sl.lkey);
  uint64_t* subkey = W.A64(W.sl.sub_v);
  const int32_t* aoff = W.A(W.sl.aoff);
  const int32_t* aadj = W.A(W.sl.aadj);
  // L_sub positions
  int n = 0;
  for (int c0 = 0; c0 < t.nL; c0 += 32) {
    int l = c0 + lane;
    bool sel = l < t.nL && llevel[l] == level;
    unsigned bal = __ballot_sync(kFull, sel);
    if (sel) {
      int j = n + __popc(bal & lanemask_lt());
      lp[j] = l;
      lkey[j] = W.gp->ukey[t.L[l]];
      if (W.p.emit) W.A(W.sl.lid)[j] = t.L[l];
    }
    n += __popc(bal);
  }
  // candidates
  int nsub = 0, nq = 0;
  for (int c0 = 0; c0 < t.nC; c0 += 32) {
    int i = c0 + lane;
    bool sel = false;
    if (i < t.nC) {
      int c = ncnt[i];
      sel = bound[i] > level && c > 0 && c < kept;
      sidx[i] = -1;
    }
    unsigned bal = __ballot_sync(kFull, sel);
    if (sel) {
      int s = nsub + __popc(bal & lanemask_lt());
      sidx[i] = s;
      subkey[s] = ckey[i];
    }
    nsub += __popc(bal);
    // candidates before x are Q
    unsigned before = __ballot_sync(kFull, sel && i < x);
    nq += __popc(before);
  }
  __syncwarp();
  if (nsub > 0) {
    const int K = words_k(n), RS = rec_stride(K);
    uint32_t* rec = reinterpret_cast<uint32_t*>(W.A(W.sl.masks));
    init_records(rec, K, nsub);
    flat_rows(
        n,
        [&](int r, int& beg, int& len) {
          int l = lp[r];
          beg = aoff[l];
          len = aoff[l + 1] - beg;
        },
        [&](bool valid, int r, int pos) {
          if (!valid) return;
          int p = aadj[pos];
          if (p < 0) return;
          int s = sidx[p];
          if (s >= 0) atomicOr(&rec[(size_t)s * RS + 1 + (r >> 5)], 1u << (r & 31));
        });
    __syncwarp();
    tier2(W, n, nsub, nq, nsub, sR, nR);
  }
  __syncwarp();
}

// A push at `level` whose child L (the `kept` rows, marked llevel == level)
// fits the bitmap tier, done without touching the level's counts: the child's
// neighbour counts are built from the kept rows alone, the child sub-problem
// goes to tier 2, and the state after finder_pop is written directly.  With
// pruning on, finder_pop leaves a candidate c of bound >= level at FREE if c
// is adjacent to a removed vertex (its count inside the kept rows is below
// its count at this level) or is x itself, and at level-1 otherwise; every
// candidate of bound >= level is FREE before the push, and candidates not
// adjacent to the kept rows are either touched (stay FREE) or irrelevant
// below this level (count 0), so only candidates adjacent to the kept rows
// change.
__device__ void t1_sparse_push(Warp& W, const T1& t, int x, int level, int kept, uint64_t sL) {
  const int lane = (int)lane_id();
  int32_t* llevel = W.A(W.sl.llevel);
  const int32_t* ncnt = W.A(W.sl.ncnt);
  int32_t* bound = W.A(W.sl.bound);
  const int32_t* cv = W.A(W.sl.cv);
  const int32_t* coff = W.A(W.sl.coff);
  const int32_t* cadj = W.A(W.sl.cadj);
  const int32_t* aoff = W.A(W.sl.aoff);
  const int32_t* aadj = W.A(W.sl.aadj);
  int32_t* cc = W.A(W.sl.fill);   // child counts, all-zero between pushes
  int32_t* sidx = W.A(W.sl.sidx); // -1 between pushes
  int32_t* tl = W.A(W.sl.tlist);
  int32_t* lp = W.A(W.sl.lp);
  uint64_t* lkey = W.A64(W.sl.lkey);
  uint64_t* subkey = W.A64(W.sl.sub_v);
  // kept rows -> lp[0..kept), with their hash keys
  int n = 0;
  {
    int rb = coff[x], re = coff[x + 1];
    for (int b0 = rb; b0 < re; b0 += 32) {
      int j = b0 + lane;
      int l = j < re ? cadj[j] : 0;
      bool sel = j < re && llevel[l] == level;
      unsigned bal = __ballot_sync(kFull, sel);
      if (sel) {
        int q = n + __popc(bal & lanemask_lt());
        lp[q] = l;
        if (q < 32 * kKMax) {
          lkey[q] = W.gp->ukey[t.L[l]];
          if (W.p.emit) W.A(W.sl.lid)[q] = t.L[l];
        }
      }
      n += __popc(bal);
    }
  }
  __syncwarp();
  // Child counts over the kept rows.  tl = candidates met (each once);
  // ent = every (candidate, row) entry met, packed p << 7 | r (r < 128), so
  // that the child's masks come from one linear pass instead of a second walk.
  int32_t* ent = W.A(W.sl.ent);
  int32_t* tcls = W.A(W.sl.tcls);
  const uint64_t* ckey = W.A64(W.sl.ckey);
  int nt = 0, ne = 0;
  int kent = 0;  // entries of the kept rows
  for (int q = lane; q < n; q += 32) kent += aoff[lp[q] + 1] - aoff[lp[q]];
  kent = warp_sum(kent);
  const int cwords = (t.nC + 31) >> 5;
  if (use_gseen(W, kent, cwords)) {
    // fire-and-forget counts and touch bits; the touched list from the bitmap
    flat_rows(
        n,
        [&](int r, int& beg, int& len) {
          int l = lp[r];
          beg = aoff[l];
          len = aoff[l + 1] - beg;
        },
        [&](bool valid, int r, int pos) {
          int p = valid ? aadj[pos] : -1;
          if (p >= 0) {
            atomicAdd(&cc[p], 1);
            atomicOr(&W.gseen[p >> 5], 1u << (p & 31));
          }
          const unsigned be = __ballot_sync(kFull, p >= 0);
          if (p >= 0) ent[ne + __popc(be & lanemask_lt())] = (p << 7) | r;
          ne += __popc(be);
        });
    __threadfence_block();
    __syncwarp();
    nt = collect_bits(W.gseen, cwords, tl, t.nC);
  } else {
    flat_rows(
        n,
        [&](int r, int& beg, int& len) {
          int l = lp[r];
          beg = aoff[l];
          len = aoff[l + 1] - beg;
        },
        [&](bool valid, int r, int pos) {
          int p = valid ? aadj[pos] : -1;
          bool first = false;
          if (p >= 0) first = count_first(W, cc, p);
          const unsigned lt = lanemask_lt();
          unsigned bal = __ballot_sync(kFull, first);
          if (first) tl[nt + __popc(bal & lt)] = p;
          nt += __popc(bal);
          unsigned be = __ballot_sync(kFull, p >= 0);
          if (p >= 0) ent[ne + __popc(be & lt)] = (p << 7) | r;
          ne += __popc(be);
        });
    counts_done(W, tl, nt);
  }
  // R of the child, maximality, and each touched candidate's class (0 none,
  // 1 Q, 2 P).  Lane-local counters keep the iterations independent, so
  // their loads overlap.
  bool ism = true;
  uint64_t sR = 0;
  unsigned long long nR = 0;
  int ncand = 0, nqc = 0;
#pragma unroll 4
  for (int q = lane; q < nt; q += 32) {
    const int p = tl[q];
    const int c = cc[p];
    const int b = bound[p];
    int cls = 0;
    if (c == kept) {
      sR += ckey[p];
      ++nR;
      if (p < x && b >= level) ism = false;
    } else if (b >= level) {
      cls = p < x ? 1 : 2;
      ++ncand;
      nqc += cls == 1;
    }
    tcls[q] = cls;
  }
  ism = __all_sync(kFull, ism);
  ncand = warp_sum(ncand);
  nqc = warp_sum(nqc);
  sR = warp_sum(sR) + t.sRtask;
  nR = warp_sum(nR) + t.nRtask;
  if (ism) {
    W.cnt += 1;
    W.hash += biclique_hash(*W.gp, sL, (uint64_t)kept, sR, nR);
    if (W.p.emit) emit_list(W.ctl, emit_dst(W.p), W.gid, n, t.L, lp);
  } else {
    W.nonmax += 1;
  }
  __syncwarp();
  if (ism && kept > 1 && ncand > 0) {
    // Destination: an export slot when idle warps want work and the child is
    // big enough by GMBE's split test, else this warp's scratch.
    const int K = words_k(n), RS = rec_stride(K);
    int slot = -1;
    if (slot_fits(W, ncand, K) && should_export(W, ncand - nqc, n, W.p.eager_share != 0)) {
      slot = lane == 0 ? slot_alloc_for(W, ncand, K) : 0;
      slot = __shfl_sync(kFull, slot, 0);
    }
    uint32_t* rec = reinterpret_cast<uint32_t*>(W.A(W.sl.masks));
    int32_t* sp = nullptr;
    if (slot >= 0) {
      sp = slot_ptr(W, slot);
      rec = reinterpret_cast<uint32_t*>(sp + kSlotRec);
      subkey = slot_subkey(sp, K, ncand);
      uint64_t* lk = reinterpret_cast<uint64_t*>(sp + kSlotLkey);
      for (int b = lane; b < n; b += 32) lk[b] = lkey[b];
      if (W.p.emit) {
        int32_t* li = sp + kSlotLid;
        const int32_t* lid = W.A(W.sl.lid);
        for (int b = lane; b < n; b += 32) li[b] = lid[b];
      }
    }
    // child indices: Q from the front, P from the back
    int nq = 0, np = 0;
    for (int b0 = 0; b0 < nt; b0 += 32) {
      int q = b0 + lane;
      const int cls = q < nt ? tcls[q] : 0;
      const int p = q < nt ? tl[q] : 0;
      unsigned bq = __ballot_sync(kFull, cls == 1);
      unsigned bp = __ballot_sync(kFull, cls == 2);
      int s = -1;
      if (cls == 1) s = nq + __popc(bq & lanemask_lt());
      if (cls == 2) s = ncand - 1 - (np + __popc(bp & lanemask_lt()));
      if (s >= 0) {
        sidx[p] = s;
        subkey[s] = ckey[p];
      }
      nq += __popc(bq);
      np += __popc(bp);
    }
    __syncwarp();
    init_records(rec, K, ncand);
#pragma unroll 4
    for (int e = lane; e < ne; e += 32) {
      const int pk = ent[e];
      const int si = sidx[pk >> 7];
      const int r = pk & 127;
      if (si >= 0) atomicOr(&rec[(size_t)si * RS + 1 + (r >> 5)], 1u << (r & 31));
    }
    __syncwarp();
    if (slot >= 0) {
      if (lane == 0) {
        uint32_t L0[4];
        full_mask(L0, n);
        slot_header(sp, K, ncand, nq, L0, sR, nR, W.gid);
      }
      if (!slot_publish(W, slot)) tier2_from_slot(W, slot);  // ring full: run it here
    } else {
      tier2(W, n, ncand, nq, ncand, sR, nR);
    }
  }
  __syncwarp();
  // state after finder_pop(x, level), then clear the child scratch
#pragma unroll 4
  for (int q = lane; q < nt; q += 32) {
    const int p = tl[q];
    if (bound[p] >= level && p != x && cc[p] == ncnt[p]) bound[p] = level - 1;
    cc[p] = 0;
    sidx[p] = -1;
  }
  for (int q = lane; q < n; q += 32) llevel[lp[q]] = level - 1;
  __syncwarp();
}

// Levels 2 .. kLevelBits + 1 of the counts tier keep a bitmap of the
// candidates the level's L meets (count != 0 there): the scan for the next
// live candidate and a recount walk its words instead of every candidate.
__device__ __forceinline__ uint32_t* level_bits(const Warp& W, int level) {
  if (level < 2 || level > kLevelBits + 1) return nullptr;
  return reinterpret_cast<uint32_t*>(W.A(W.sl.lbits)) +
         (size_t)(level - 2) * (size_t)((W.sl.capC + 31) >> 5);
}

__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(kFull, v, o));
  return v;
}

// First candidate i in [start, end) with bound[i] > level-1 and ncnt[i] != 0
// (src/IterFinderGpu.cu:26-34), or -1.  bits, when given, holds the
// candidates with ncnt != 0.
__device__ __forceinline__ int t1_next_live(const int32_t* bound, const int32_t* ncnt,
                                            const uint32_t* bits, int start, int end, int level) {
  const int lane = (int)lane_id();
  if (!bits) {
    for (int b0 = start; b0 < end; b0 += 32) {
      const int i = b0 + lane;
      const bool ok = i < end && bound[i] > level - 1 && ncnt[i] != 0;
      const unsigned bal = __ballot_sync(kFull, ok);
      if (bal) return b0 + __ffs(bal) - 1;
    }
    return -1;
  }
  if (start >= end) return -1;
  const int w0 = start >> 5, wend = (end + 31) >> 5;
  for (int wb = w0; wb < wend; wb += 32) {
    const int w = wb + lane;
    uint32_t m = w < wend ? bits[w] : 0u;
    if (w == w0) m &= ~0u << (start & 31);
    if (w == wend - 1 && (end & 31)) m &= (1u << (end & 31)) - 1u;
    int first = -1;
    while (m) {
      const int i = (w << 5) + __ffs(m) - 1;
      if (bound[i] > level - 1) {
        first = i;
        break;
      }
      m &= m - 1;
    }
    const unsigned bal = __ballot_sync(kFull, first >= 0);
    if (bal) return __shfl_sync(kFull, first, __ffs(bal) - 1);
  }
  return -1;
}

// Counts-tier child export.  A push at `level` of candidate x whose new L
// (the `kept` rows, llevel == level) is too large for the bitmap tier
// descends in place; when warps wait for work the child goes to one of them
// instead, as vertex lists in a slot: L' = the kept rows' vertices, C' = the
// candidates live below this level (bound > level) with 0 < count < kept,
// in index order (those before x are its Q), and the R sum and size of the
// push.  Every bound of C' is free at the child's first level (a bound above
// `level` is FREE or TOUCHED there), so the importer starts from a clean
// frame, and the child's levels leave this level's state as they found it:
// the exporter pops x at once.  nbits holds the candidates the kept rows
// meet (the bitmap of level + 1).  Slot: header of 16 words {|L'|, |C'|,
// |Q'|, graph, sR (2 words), |R|}, then L' ids, then C' ids.
constexpr int kFrameHdr = 16;

// Whether a counts-tier child of `kept` rows (`kent` entries) may be shared
// out now: slots exist, every warp has room for it, warps wait for work.
__device__ __forceinline__ bool t1_export_wanted(Warp& W, int kept, long long kent) {
  if (!W.p.share_counts || (W.nslot == 0 && W.nbig == 0)) return false;
  if (kept > W.import_l || kent > (long long)W.import_s) return false;
  return export_demand(W) != 0;
}

__device__ bool t1_try_export(Warp& W, const T1& t, int x, int level, int kept, long long kent,
                              uint64_t sR, uint64_t nR, const uint32_t* nbits) {
  const int lane = (int)lane_id();
  const int32_t* bound = W.A(W.sl.bound);
  const int32_t* ncnt = W.A(W.sl.ncnt);
  const int32_t* cv = W.A(W.sl.cv);
  const int32_t* coff = W.A(W.sl.coff);
  const int32_t* cadj = W.A(W.sl.cadj);
  const int32_t* llevel = W.A(W.sl.llevel);
  const int cwords = (t.nC + 31) >> 5;
  int m = 0, mq = 0;
  for (int w0 = 0; w0 < cwords; w0 += 32) {
    const int w = w0 + lane;
    uint32_t b = w < cwords ? nbits[w] : 0u;
    while (b) {
      const int p = (w << 5) + __ffs(b) - 1;
      if (bound[p] > level && ncnt[p] < kept) {
        ++m;
        mq += p < x;
      }
      b &= b - 1;
    }
  }
  m = warp_sum(m);
  mq = warp_sum(mq);
  if (m == 0 || m > W.import_cap || !should_export(W, m - mq, kept)) return false;
  const long long words = kFrameHdr + (long long)kept + m;
  int slot = -1;
  if (lane == 0) {
    if (words <= kSlotWords) slot = slot_alloc(W);
    if (slot < 0 && words <= kBigSlotWords) {
      const int b = bits_alloc(W.big_bits, W.nbig);
      if (b >= 0) slot = W.nslot + b;
    }
  }
  slot = __shfl_sync(kFull, slot, 0);
  if (slot < 0) return false;
  int32_t* sp = slot_ptr(W, slot);
  // L' ids: the kept rows, from x's row of cadj
  int nl = 0;
  for (int j0 = coff[x]; j0 < coff[x + 1]; j0 += 32) {
    const int j = j0 + lane;
    const int l = j < coff[x + 1] ? cadj[j] : 0;
    const bool sel = j < coff[x + 1] && llevel[l] == level;
    const unsigned bal = __ballot_sync(kFull, sel);
    if (sel) sp[kFrameHdr + nl + __popc(bal & lanemask_lt())] = t.L[l];
    nl += __popc(bal);
  }
  // C' ids in index order: lane k takes word k of each round
  int32_t* cdst = sp + kFrameHdr + kept;
  int o = 0;
  for (int w0 = 0; w0 < cwords; w0 += 32) {
    const int w = w0 + lane;
    uint32_t b = w < cwords ? nbits[w] : 0u;
    uint32_t keep = 0u;
    for (uint32_t bb = b; bb; bb &= bb - 1) {
      const int bit = __ffs(bb) - 1;
      const int p = (w << 5) + bit;
      if (bound[p] > level && ncnt[p] < kept) keep |= 1u << bit;
    }
    int tot;
    int at = o + warp_excl_scan(__popc(keep), &tot);
    for (; keep; keep &= keep - 1) cdst[at++] = cv[(w << 5) + __ffs(keep) - 1];
    o += tot;
  }
  if (lane == 0) {
    sp[0] = kept;
    sp[1] = m;
    sp[2] = mq;
    sp[3] = W.gid;
    *reinterpret_cast<uint64_t*>(sp + 4) = sR;
    sp[6] = (int32_t)nR;
  }
  if (slot_publish(W, slot, 1)) {
    W.splits += 1;
    return true;
  }
  if (lane == 0) slot_free(W, slot);
  __syncwarp();
  return false;
}

__device__ void tier1_run(Warp& W, const T1& t) {
  const int lane = (int)lane_id();
  int32_t* llevel = W.A(W.sl.llevel);
  int32_t* ncnt = W.A(W.sl.ncnt);
  int32_t* bound = W.A(W.sl.bound);
  int32_t* stack = W.A(W.sl.stack);
  int32_t* lent = W.A(W.sl.lent);
  const uint64_t* ckey = W.A64(W.sl.ckey);
  const int32_t* coff = W.A(W.sl.coff);
  const int32_t* cadj = W.A(W.sl.cadj);
  const int32_t* aoff = W.A(W.sl.aoff);
  const int32_t* aadj = W.A(W.sl.aadj);
  const bool emitting = W.p.emit != nullptr;
  const int t2max = W.gp->tier2_max_l;
  const int cwords = (t.nC + 31) >> 5;

  // The level bitmaps start clear (a task that ended early may leave bits).
  for (int lv = 2; lv <= kLevelBits + 1; ++lv) {
    uint32_t* b = level_bits(W, lv);
    for (int w = lane; w < cwords; w += 32) b[w] = 0u;
  }
  if (lane == 0) {
    stack[0] = t.nq;
    lent[0] = aoff[t.nL];
  }
  __syncwarp();
  int level = 1;
  unsigned steps = 0;
  while (level != 0) {
    // The stop flag is a global load the whole warp waits for: look at it on
    // the first step and every 64th after.
    if ((steps++ & 63u) == 0u && must_stop(W)) return;
    const int end = level == 1 ? t.nend : t.nC;  // the first level may push a part only
    int cur = t1_next_live(bound, ncnt, level_bits(W, level), stack[level - 1], end, level);
    if (cur >= 0) {
      // ---- finder_push (src/IterFinderGpu.h:206-264) ----
      W.pushes += 1;
      int kept = 0;
      uint64_t sL = 0;
      long long kent = 0;                 // entries of the kept rows
      unsigned long long best = ~0ULL;    // (row length << 32) | position of the shortest kept row
      int rb = coff[cur], re = coff[cur + 1];
      for (int j = rb + lane; j < re; j += 32) {
        int l = cadj[j];
        if (llevel[l] == level - 1) {
          llevel[l] = level;
          ++kept;
          sL += W.gp->ukey[t.L[l]];
          const int len = aoff[l + 1] - aoff[l];
          kent += len;
          best = min(best, ((unsigned long long)(unsigned)len << 32) | (unsigned)l);
        }
      }
      kept = warp_sum(kept);
      sL = warp_sum(sL);
      kent = warp_sum(kent);
      best = warp_min_u64(best);
      __syncwarp();
      if (W.p.prune && kept <= t2max) {
        t1_sparse_push(W, t, cur, level, kept, sL);
        if (lane == 0) stack[level - 1] = cur + 1;
        __syncwarp();
        continue;
      }
      // Counts over the kept rows: subtract the removed rows, or clear the
      // level's counts and add the kept rows, whichever walks less.
      const uint32_t* pbits = level_bits(W, level);
      const long long rent = (long long)lent[level - 1] - kent;
      const long long clear_cost = pbits ? (long long)cwords : (long long)t.nC;
      if (clear_cost + kent < rent) {
        if (pbits) {
          for (int w = lane; w < cwords; w += 32) {
            uint32_t m = pbits[w];
            while (m) {
              ncnt[(w << 5) + __ffs(m) - 1] = 0;
              m &= m - 1;
            }
          }
        } else {
          for (int i = lane; i < t.nC; i += 32) ncnt[i] = 0;
        }
        __syncwarp();
        t1_rows_of(W, cur, level, [&](bool valid, int, int pos) {
          if (!valid) return;
          int p = aadj[pos];
          if (p >= 0) atomicAdd(&ncnt[p], 1);
        });
      } else {
        t1_rows_at_level(W, t, level - 1, [&](bool valid, int, int pos) {
          if (!valid) return;
          int p = aadj[pos];
          if (p >= 0) atomicSub(&ncnt[p], 1);
        });
      }
      __syncwarp();
      // Maximality (src/IterFinderGpu.h:252-261): a candidate covering the new
      // L is adjacent to every kept row, the shortest one included, so only
      // that row's candidates are examined.
      bool ism = true;
      uint64_t sR = 0;
      unsigned long long nR = 0;
      {
        const int lstar = (int)(best & 0xffffffffu);
        const int mb = aoff[lstar], me = aoff[lstar + 1];
        for (int j = mb + lane; j < me; j += 32) {
          const int i = aadj[j];
          if (i >= 0 && ncnt[i] == kept) {
            sR += ckey[i];
            ++nR;
            int b = bound[i];
            if (i < cur && b >= level) ism = false;
            else if (b > level) bound[i] = level;
          }
        }
      }
      ism = __all_sync(kFull, ism);
      sR = warp_sum(sR) + t.sRtask;
      nR = warp_sum(nR) + t.nRtask;
      if (ism) {
        W.cnt += 1;
        W.hash += biclique_hash(*W.gp, sL, (uint64_t)kept, sR, nR);
        if (emitting)
          emit_level(W.ctl, emit_dst(W.p), W.gid, kept, t.nL, llevel, level, t.L);
      } else {
        W.nonmax += 1;
      }
      __syncwarp();
      if (ism && kept > 1) {
        if (kept <= t2max) {
          t1_handoff(W, t, cur, level, kept, sR, nR);
        } else {
          uint32_t* nbits = level_bits(W, level + 1);
          // The candidates the kept rows meet, as a bitmap: the next level's
          // own one, or (deeper levels) the warp's global touch bitmap, built
          // only when the child may be shared out.
          uint32_t* cbits = nbits;
          const bool want = t1_export_wanted(W, kept, kent);
          if (!cbits && want) cbits = W.gseen;
          if (cbits) {
            t1_rows_of(W, cur, level, [&](bool valid, int, int pos) {
              if (!valid) return;
              const int p = aadj[pos];
              if (p >= 0) atomicOr(&cbits[p >> 5], 1u << (p & 31));
            });
            __threadfence_block();
            __syncwarp();
          }
          const bool exported =
              want && cbits && t1_try_export(W, t, cur, level, kept, kent, sR, nR, cbits);
          if (cbits && (exported || cbits != nbits)) {
            // back to clear: a shared-out child's level bitmap, or the touch bitmap
            t1_rows_of(W, cur, level, [&](bool valid, int, int pos) {
              if (!valid) return;
              const int p = aadj[pos];
              if (p >= 0) cbits[p >> 5] = 0u;
            });
            __syncwarp();
          }
          if (exported) {
            // shared out: pop x here
          } else {
            if (lane == 0) {
              stack[level - 1] = cur;
              stack[level] = cur + 1;
              lent[level] = (int32_t)kent;
            }
            __syncwarp();
            ++level;
            continue;
          }
        }
      }
      if (lane == 0) stack[level - 1] = cur + 1;
      __syncwarp();
      t1_pop(W, t, cur, level);
    } else {
      --level;
      if (level > 0) {
        cur = stack[level - 1];
        __syncwarp();
        uint32_t* cbits = level_bits(W, level + 1);
        if (cbits) {  // the finished level's bitmap back to clear
          t1_rows_of(W, cur, level, [&](bool valid, int, int pos) {
            if (!valid) return;
            const int p = aadj[pos];
            if (p >= 0) cbits[p >> 5] = 0u;
          });
          __syncwarp();
        }
        t1_pop(W, t, cur, level);
        if (lane == 0) stack[level - 1] = cur + 1;
        __syncwarp();
      }
    }
  }
}

// Runs a counts-tier child exported by t1_try_export: the frame is rebuilt
// from the vertex lists (local adjacency from the graph's U -> V rows, the
// counts of each candidate inside L'), then the counts tier runs it from its
// first level.  The child's own biclique was counted by the exporter.
__device__ void tier1_from_slot(Warp& W, int slot) {
  const int lane = (int)lane_id();
  int32_t* sp = slot_ptr(W, slot);
  volatile const int32_t* vh = sp;
  const int n = vh[0], m = vh[1], nq = vh[2];
  const int32_t gid = vh[3];
  const uint64_t sR = (uint64_t)(uint32_t)vh[4] | ((uint64_t)(uint32_t)vh[5] << 32);
  const uint64_t nR = (uint32_t)vh[6];
  int32_t* lv = W.A(W.sl.lv);
  int32_t* cv = W.A(W.sl.cv);
  const bool fits = n <= W.sl.capL && m <= W.sl.capC;
  if (fits) {
    const unsigned* src = reinterpret_cast<const unsigned*>(sp + kFrameHdr);
    for (int i = lane; i < n; i += 32) lv[i] = (int32_t)__ldcg(src + i);
    for (int i = lane; i < m; i += 32) cv[i] = (int32_t)__ldcg(src + n + i);
  }
  __syncwarp();
  if (lane == 0) slot_free(W, slot);
  __syncwarp();
  if (!fits) {
    set_status(W.ctl, kStCapacity, ((unsigned long long)4 << 32) | (unsigned)m);
    return;
  }
  W.gid = gid;
  W.gp = graph_at(W, gid);
  const DevGraph& g = *W.gp;
  int32_t* map = W.A(W.sl.map);
  int32_t* aoff = W.A(W.sl.aoff);
  int32_t* aadj = W.A(W.sl.aadj);
  int32_t* ent = W.A(W.sl.ent);
  int32_t* ncnt = W.A(W.sl.ncnt);
  int32_t* bound = W.A(W.sl.bound);
  int32_t* coff = W.A(W.sl.coff);
  int32_t* fill = W.A(W.sl.fill);
  int32_t* cadj = W.A(W.sl.cadj);
  int32_t* sidx = W.A(W.sl.sidx);
  int32_t* llevel = W.A(W.sl.llevel);
  uint64_t* ckey = W.A64(W.sl.ckey);
  uint64_t t0 = globaltimer_ns();
  int run = 0;
  for (int c0 = 0; c0 < n; c0 += 32) {
    const int l = c0 + lane;
    const int d = l < n ? g.rev_off[lv[l] + 1] - g.rev_off[lv[l]] : 0;
    int tot;
    const int ex = warp_excl_scan(d, &tot);
    if (l < n) aoff[l] = run + ex;
    run += tot;
  }
  if (lane == 0) aoff[n] = run;
  if (run > W.sl.capS) {
    set_status(W.ctl, kStCapacity, ((unsigned long long)5 << 32) | (unsigned)run);
    return;
  }
  for (int i = lane; i < m; i += 32) {
    map[cv[i]] = i + 1;
    ncnt[i] = 0;
    bound[i] = kFree;
    fill[i] = 0;
    sidx[i] = -1;
    ckey[i] = g.vkey[cv[i]];
  }
  for (int l = lane; l < n; l += 32) llevel[l] = 0;
  __threadfence_block();
  __syncwarp();
  flat_rows(
      n,
      [&](int r, int& beg, int& len) {
        const int u = lv[r];
        beg = g.rev_off[u];
        len = g.rev_off[u + 1] - beg;
      },
      [&](bool valid, int r, int pos) {
        if (!valid) return;
        const int u = lv[r];
        const int off = aoff[r] + (pos - g.rev_off[u]);
        const int p = map[__ldg(g.rev_col + pos)] - 1;
        aadj[off] = p;
        ent[off] = r;
        if (p >= 0) atomicAdd(&ncnt[p], 1);
      });
  __threadfence_block();
  __syncwarp();
  {
    int acc = 0;
    for (int c0 = 0; c0 < m; c0 += 32) {
      const int i = c0 + lane;
      const int c = i < m ? ncnt[i] : 0;
      int tot;
      const int ex = warp_excl_scan(c, &tot);
      if (i < m) coff[i] = acc + ex;
      acc += tot;
    }
    if (lane == 0) coff[m] = acc;
  }
  __syncwarp();
  for (int j0 = 0; j0 < run; j0 += 128) {
    int pp[4], rr[4], ss[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int j = j0 + k * 32 + lane;
      pp[k] = j < run ? aadj[j] : -1;
      rr[k] = j < run ? ent[j] : 0;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) ss[k] = pp[k] >= 0 ? atomicAdd(&fill[pp[k]], 1) : 0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (pp[k] >= 0) cadj[coff[pp[k]] + ss[k]] = rr[k];
  }
  __syncwarp();
  for (int i = lane; i < m; i += 32) fill[i] = 0;
  __syncwarp();
  T1 t1;
  t1.L = lv;
  t1.nL = n;
  t1.nC = m;
  t1.nq = nq;
  t1.nend = m;
  t1.sRtask = sR;
  t1.nRtask = nR;
  const uint64_t t1s = globaltimer_ns();
  const uint64_t t2_before = W.ns_t2;
  tier1_run(W, t1);
  W.ns_t1 += (globaltimer_ns() - t1s) - (W.ns_t2 - t2_before);
  (void)t0;
  __syncwarp();
  for (int i = lane; i < m; i += 32) map[cv[i]] = 0;
  __syncwarp();
}

// ---------------------------------------------------------------------------
// Queue (bounded MPMC ring; replaces WorkList<LargeTask>, src/WorkList.cuh).
//
// Position gp lives in slot gp % cap during round gp / cap.  A slot's state
// word is 2*round while it is free for that round's producer and 2*round+1
// once the task is written; the consumer of position h hands the slot to the
// next round by writing 2*(h/cap)+2.  q_used (reserved, not yet released
// positions) never exceeds cap, so a producer only ever waits for a consumer
// that has already claimed the older position and is reading it.
__device__ __forceinline__ unsigned long long slot_free_tag(unsigned long long gp, int cap) {
  return 2ULL * (gp / (unsigned long long)cap);
}

__device__ bool queue_pop(Warp& W, Task* out) {
  // lane 0 only
  EnumCtl* ctl = W.ctl;
  volatile unsigned long long* vh = &ctl->q_head;
  volatile unsigned long long* vt = &ctl->q_tail;
  unsigned long long h = *vh;
  if (h >= *vt) return false;
  if (atomicCAS(&ctl->q_head, h, h + 1) != h) return false;
  const int cap = W.p.queue_cap;
  unsigned long long slot = h % (unsigned long long)cap;
  volatile unsigned long long* st = W.q_seq + slot;
  const unsigned long long full = slot_free_tag(h, cap) + 1;
  int64_t spins = 0;
  while (*st != full) {
    if (++spins > W.p.slot_spin_limit) {
      set_status(ctl, kStQueue, h);
      return false;
    }
    __nanosleep(64);
  }
  __threadfence();
  volatile int32_t* src = reinterpret_cast<volatile int32_t*>(W.q_tasks + slot);
  out->v[0] = src[0];
  out->v[1] = src[1];
  out->v[2] = src[2];
  out->v[3] = src[3];
  out->graph = src[4];
  out->part = src[5];
  out->parts = src[6];
  __threadfence();
  atomicExch(W.q_seq + slot, full + 1);  // free for round h/cap + 1
  atomicAdd(&ctl->q_used, (unsigned long long)-1LL);
  return true;
}

// Queues n tasks, task i (0 <= i < n) made by make(i); false if the ring is
// full (then nothing is queued).
template <typename Make>
__device__ bool queue_push_n(Warp& W, unsigned long long n, Make make) {
  const int lane = (int)lane_id();
  EnumCtl* ctl = W.ctl;
  const int cap = W.p.queue_cap;
  unsigned long long pos = 0;
  int ok = 0;
  if (lane == 0) {
    unsigned long long used = atomicAdd(&ctl->q_used, n);
    if (used + n > (unsigned long long)cap) {
      atomicAdd(&ctl->q_used, (unsigned long long)(-(long long)n));
    } else {
      atomicAdd(&ctl->pending, n);
      graph_spawned(W, n);
      pos = atomicAdd(&ctl->q_tail, n);
      ok = 1;
    }
  }
  ok = __shfl_sync(kFull, ok, 0);
  if (!ok) return false;
  pos = __shfl_sync(kFull, pos, 0);
  for (unsigned long long i = lane; i < n; i += 32) {
    unsigned long long gp = pos + i;
    unsigned long long slot = gp % (unsigned long long)cap;
    volatile unsigned long long* st = W.q_seq + slot;
    const unsigned long long free_tag = slot_free_tag(gp, cap);
    int64_t spins = 0;
    bool ready = true;
    while (*st != free_tag) {
      if (++spins > W.p.slot_spin_limit) {
        set_status(ctl, kStQueue, gp);
        ready = false;
        break;
      }
      __nanosleep(64);
    }
    if (!ready) continue;  // the run is aborting; the slot stays unwritten
    W.q_tasks[slot] = make((int)i);
    __threadfence();
    atomicExch(W.q_seq + slot, free_tag + 1);
  }
  __syncwarp();
  return true;
}

// Pushes children task + {cv[i]} for i in [nq, nC); false if the ring is full.
__device__ bool queue_push_children(Warp& W, const Task& t, int k, int nq, int nC) {
  const int32_t* cv = W.A(W.sl.cv);
  return queue_push_n(W, (unsigned long long)(nC - nq), [&](int i) {
    Task c = t;
    c.v[k] = cv[nq + i];
    c.part = c.parts = 0;
    return c;
  });
}

// Pushes parts 1 .. m-1 of root task t; false if the ring is full.
__device__ bool queue_push_parts(Warp& W, const Task& t, int m) {
  return queue_push_n(W, (unsigned long long)(m - 1), [&](int i) {
    Task c = t;
    c.part = i + 1;
    c.parts = m;
    return c;
  });
}

// Parts 1 .. m-1 of a listed big root (lane-uniform): a part record that only
// big warps claim from (the other warps' scratch cannot hold the root).
// They count as pending before the record becomes visible.  False if the
// record list is full (the root then runs whole).
__device__ bool big_parts_push(Warp& W, int v, int m) {
  int ok = 0;
  if (lane_id() == 0) {
    const unsigned long long i = atomicAdd(&W.ctl->n_big_parts, 1ULL);
    if (i < (unsigned long long)W.p.big_parts_cap) {
      atomicAdd(&W.ctl->pending, (unsigned long long)(m - 1));
      int32_t* r = W.p.big_parts + 4 * i;
      r[0] = v;
      r[1] = m;
      r[2] = 1;  // part 0 runs on this warp
      __threadfence();
      atomicExch(&r[3], 1);
      ok = 1;
    }
  }
  return __shfl_sync(kFull, ok, 0) != 0;
}

// Claims a part of a listed big root (lane 0 of a big warp).
__device__ bool big_parts_claim(Warp& W, Task* t) {
  EnumCtl* c = W.ctl;
  const unsigned long long n = min(*(volatile unsigned long long*)&c->n_big_parts,
                                   (unsigned long long)W.p.big_parts_cap);
  for (unsigned long long i = *(volatile unsigned long long*)&c->big_parts_head; i < n; ++i) {
    int32_t* r = W.p.big_parts + 4 * i;
    if (*(volatile int32_t*)&r[3] == 0) continue;  // being written
    const int m = *(volatile int32_t*)&r[1];
    if (*(volatile int32_t*)&r[2] < m) {
      const int j = atomicAdd(&r[2], 1);
      if (j < m) {
        t->v[0] = *(volatile int32_t*)&r[0];
        t->v[1] = t->v[2] = t->v[3] = -1;
        t->graph = 0;
        t->part = j;
        t->parts = m;
        t->pad = 0;
        return true;
      }
    }
    // exhausted: move the head past it (another warp may have done so)
    atomicCAS(&c->big_parts_head, i, i + 1);
  }
  return false;
}

// Pushes one task (lane-uniform); false if the ring is full.
__device__ bool queue_push_one(Warp& W, const Task& t) {
  const int lane = (int)lane_id();
  EnumCtl* ctl = W.ctl;
  const int cap = W.p.queue_cap;
  int ok = 0;
  if (lane == 0) {
    unsigned long long used = atomicAdd(&ctl->q_used, 1ULL);
    if (used + 1 > (unsigned long long)cap) {
      atomicAdd(&ctl->q_used, (unsigned long long)-1LL);
    } else {
      atomicAdd(&ctl->pending, 1ULL);
      graph_spawned(W, 1ULL);
      unsigned long long gp = atomicAdd(&ctl->q_tail, 1ULL);
      unsigned long long slot = gp % (unsigned long long)cap;
      volatile unsigned long long* st = W.q_seq + slot;
      const unsigned long long free_tag = slot_free_tag(gp, cap);
      int64_t spins = 0;
      ok = 1;
      while (*st != free_tag) {
        if (++spins > W.p.slot_spin_limit) {
          set_status(ctl, kStQueue, gp);
          ok = 2;
          break;
        }
        __nanosleep(64);
      }
      if (ok == 1) {
        W.q_tasks[slot] = t;
        __threadfence();
        atomicExch(W.q_seq + slot, free_tag + 1);
      }
    }
  }
  ok = __shfl_sync(kFull, ok, 0);
  return ok != 0;  // 2: the run is aborting; the task counts as handed over
}

// ---------------------------------------------------------------------------
// Task set-up (IterFinderWithMultipleVertex) and dispatch.
__device__ void run_task(Warp& W, const Task& t) {
  const int lane = (int)lane_id();
  const DevGraph& g = *W.gp;
  int k = 1;
  while (k < 4 && t.v[k] >= 0) ++k;
  const int last = t.v[k - 1];
  int32_t* map = W.A(W.sl.map);
  int32_t* touched = W.A(W.sl.touched);
  int32_t* lv = W.A(W.sl.lv);

  // ---- L = common neighbours of the task vertices ----
  const int32_t* L;
  int nL;
  if (k == 1) {
    L = g.col + g.row_off[last];
    nL = g.row_off[last + 1] - g.row_off[last];
  } else {
    // Intersect: probe the smallest row against the others.
    int best = 0, bestlen = 0x7fffffff;
    for (int i = 0; i < k; ++i) {
      int len = g.row_off[t.v[i] + 1] - g.row_off[t.v[i]];
      if (len < bestlen) {
        bestlen = len;
        best = i;
      }
    }
    const int32_t* sm = g.col + g.row_off[t.v[best]];
    int n = 0;
    for (int b0 = 0; b0 < bestlen; b0 += 32) {
      int j = b0 + lane;
      bool in = j < bestlen;
      int u = in ? __ldg(sm + j) : 0;
      for (int i = 0; i < k && in; ++i) {
        if (i == best) continue;
        const int32_t* row = g.col + g.row_off[t.v[i]];
        in = contains_sorted(row, g.row_off[t.v[i] + 1] - g.row_off[t.v[i]], u);
      }
      unsigned bal = __ballot_sync(kFull, in);
      if (in) lv[n + __popc(bal & lanemask_lt())] = u;
      n += __popc(bal);
    }
    __syncwarp();
    L = lv;
    nL = n;
  }
  if (nL == 0) return;
  if (nL > W.sl.capL) {
    set_status(W.ctl, kStCapacity, ((unsigned long long)1 << 32) | (unsigned)nL);
    return;
  }

  // ---- two-hop multiset: counts in the per-warp dense map ----
  int32_t* aoff = W.A(W.sl.aoff);
  {
    int run = 0;
    for (int c0 = 0; c0 < nL; c0 += 32) {
      int l = c0 + lane;
      int d = 0;
      if (l < nL) {
        int u = L[l];
        d = g.rev_off[u + 1] - g.rev_off[u];
      }
      int tot;
      int ex = warp_excl_scan(d, &tot);
      if (l < nL) aoff[l] = run + ex;
      run += tot;
    }
    if (lane == 0) aoff[nL] = run;
    if (run > W.sl.capS) {
      set_status(W.ctl, kStCapacity, ((unsigned long long)2 << 32) | (unsigned)run);
      return;
    }
  }
  __syncwarp();
  int nt = 0;
  const int vwords = (g.nV + 31) >> 5;
  if (use_gseen(W, aoff[nL], vwords)) {
    // Large set-up without the shared bitmap: fire-and-forget counts and
    // touch bits, then the touched list in id order from the bitmap.
    flat_rows(
        nL,
        [&](int r, int& beg, int& len) {
          int u = L[r];
          beg = g.rev_off[u];
          len = g.rev_off[u + 1] - beg;
        },
        [&](bool valid, int, int pos) {
          if (!valid) return;
          const int w = __ldg(g.rev_col + pos);
          atomicAdd(&map[w], 1);
          atomicOr(&W.gseen[w >> 5], 1u << (w & 31));
        });
    __threadfence_block();
    __syncwarp();
    nt = collect_bits(W.gseen, vwords, touched, W.sl.capC);
  } else {
    flat_rows(
        nL,
        [&](int r, int& beg, int& len) {
          int u = L[r];
          beg = g.rev_off[u];
          len = g.rev_off[u + 1] - beg;
        },
        [&](bool valid, int, int pos) {
          int w = valid ? __ldg(g.rev_col + pos) : 0;
          bool isnew = valid && count_first(W, map, w);
          unsigned bal = __ballot_sync(kFull, isnew);
          if (isnew && nt + __popc(bal & lanemask_lt()) < W.sl.capC)
            touched[nt + __popc(bal & lanemask_lt())] = w;
          nt += __popc(bal);
        });
    counts_done(W, touched, min(nt, W.sl.capC));
  }
  if (nt > W.sl.capC) {
    // Vertices beyond the touched list's room keep counts: clear the whole
    // map (the launch is failing; this keeps the invariant for the record).
    set_status(W.ctl, kStCapacity, ((unsigned long long)3 << 32) | (unsigned)nt);
    for (int i = lane; i < g.nV; i += 32) map[i] = 0;
    __syncwarp();
    return;
  }

  // ---- classify: R (count == |L|), Q (w < last), P (w > last) ----
  int32_t* cv = W.A(W.sl.cv);
  int32_t* ncnt = W.A(W.sl.ncnt);
  int32_t* bound = W.A(W.sl.bound);
  uint64_t sR = 0;
  unsigned long long nR = 0;
  int nq = 0, np = 0, nend = 0;
  int viol_first = 0x7fffffff;  // smallest R vertex below `last` (maximality witnesses)
  int nC = 0;
  // C is laid out [Q | P before this part | P of this part | P after it]; a
  // task that is not a part has only the middle P group.  The first level
  // pushes the candidates of this part; those before it act as Q, those after
  // it stay candidates of the children.
  int part = t.part, parts = t.parts;
  int cntQ = 0, cntPre = 0, cntIn = 0;
  {
    int cntC = 0;
    bool r_below = false;
    for (int b0 = 0; b0 < nt; b0 += 32) {
      int i = b0 + lane;
      bool valid = i < nt;
      int w = valid ? touched[i] : 0;
      int c = valid ? map[w] : 0;
      bool isC = valid && c != nL;
      cntC += __popc(__ballot_sync(kFull, isC));
      cntQ += __popc(__ballot_sync(kFull, isC && w < last));
      r_below |= __ballot_sync(kFull, valid && c == nL && w < last) != 0u;
    }
    nC = cntC;
    const int np_all = cntC - cntQ;
    // A heavy maximal root is split into parts before its C is laid out.
    // Its first level costs about |P| pushes, each a pass over all of C.
    if (k == 1 && parts == 0 && !r_below && W.p.range_work > 0 &&
        np_all >= 2 * W.p.range_chunk &&
        (long long)np_all * cntC > (long long)W.p.range_work) {
      const int m = min((np_all + W.p.range_chunk - 1) / W.p.range_chunk, kMaxParts);
      // A listed big root's parts go to big warps only; other roots' parts
      // fit every warp and take the common queue.
      const bool big_root = W.p.n_big_warps > 0 && W.p.big_flag[last];
      if (big_root ? big_parts_push(W, last, m) : queue_push_parts(W, t, m)) {
        part = 0;
        parts = m;
        W.splits += 1;
      }
    }
    if (parts > 1) {
      for (int b0 = 0; b0 < nt; b0 += 32) {
        int i = b0 + lane;
        bool valid = i < nt;
        int w = valid ? touched[i] : 0;
        bool isP = valid && map[w] != nL && w > last;
        int b = isP ? part_of(w, parts) : 0;
        cntPre += __popc(__ballot_sync(kFull, isP && b < part));
        cntIn += __popc(__ballot_sync(kFull, isP && b == part));
      }
    } else {
      cntIn = np_all;
    }
  }
  {
    int oQ = 0, oPre = cntQ, oIn = cntQ + cntPre, oPost = cntQ + cntPre + cntIn;
    for (int b0 = 0; b0 < nt; b0 += 32) {
      int i = b0 + lane;
      bool valid = i < nt;
      int w = valid ? touched[i] : 0;
      int c = valid ? map[w] : 0;
      bool isR = valid && c == nL;
      bool isQ = valid && !isR && w < last;
      bool isP = valid && !isR && w > last;
      int b = (isP && parts > 1) ? part_of(w, parts) : part;
      bool isPre = isP && b < part, isIn = isP && b == part, isPost = isP && b > part;
      if (isR) {
        sR += g.vkey[w];
        ++nR;
        if (w < last) viol_first = min(viol_first, w);
      }
      unsigned bq = __ballot_sync(kFull, isQ);
      unsigned bpre = __ballot_sync(kFull, isPre);
      unsigned bin = __ballot_sync(kFull, isIn);
      unsigned bpost = __ballot_sync(kFull, isPost);
      const unsigned lt = lanemask_lt();
      int pos = -1;
      if (isQ) pos = oQ + __popc(bq & lt);
      if (isPre) pos = oPre + __popc(bpre & lt);
      if (isIn) pos = oIn + __popc(bin & lt);
      if (isPost) pos = oPost + __popc(bpost & lt);
      if (pos >= 0) {
        cv[pos] = w;
        ncnt[pos] = c;
        bound[pos] = kFree;
        map[w] = pos + 1;
      } else if (valid) {
        map[w] = 0;
      }
      oQ += __popc(bq);
      oPre += __popc(bpre);
      oIn += __popc(bin);
      oPost += __popc(bpost);
    }
    nq = cntQ + cntPre;  // first P position this task pushes
    np = cntIn;
    nend = nq + cntIn;
    W.shape = (unsigned long long)(unsigned)nC | ((unsigned long long)(part & 0xffff) << 32) |
              ((unsigned long long)(parts & 0xffff) << 48);
  }
  sR = warp_sum(sR);
  nR = warp_sum(nR);
  viol_first = warp_min_i(viol_first);
  __syncwarp();

  // ---- maximality of the task (src/IterFinderGpu.cu:800-822) ----
  bool ism = true;
  if (viol_first != 0x7fffffff) {
    if (k == 1) {
      ism = false;  // R[0] != root
    } else {
      // Every R vertex below `last` must already cover L_parent.
      int32_t* lp = W.A(W.sl.lp);
      const int32_t* Lpar;
      int nLp;
      if (k == 2) {
        Lpar = g.col + g.row_off[t.v[0]];
        nLp = g.row_off[t.v[0] + 1] - g.row_off[t.v[0]];
      } else {
        const int32_t* r0 = g.col + g.row_off[t.v[0]];
        int len0 = g.row_off[t.v[0] + 1] - g.row_off[t.v[0]];
        int n = 0;
        for (int b0 = 0; b0 < len0; b0 += 32) {
          int j = b0 + lane;
          bool in = j < len0;
          int u = in ? __ldg(r0 + j) : 0;
          for (int i = 1; i < k - 1 && in; ++i)
            in = contains_sorted(g.col + g.row_off[t.v[i]],
                                 g.row_off[t.v[i] + 1] - g.row_off[t.v[i]], u);
          unsigned bal = __ballot_sync(kFull, in);
          if (in) lp[n + __popc(bal & lanemask_lt())] = u;
          n += __popc(bal);
        }
        __syncwarp();
        Lpar = lp;
        nLp = n;
      }
      for (int b0 = 0; b0 < nt && ism; b0 += 32) {
        int i = b0 + lane;
        int w = i < nt ? touched[i] : 0;
        bool cand = i < nt && w < last && map[w] == 0;  // R vertex below last
        // (map[w] == 0 marks R after classification)
        unsigned bal = __ballot_sync(kFull, cand);
        while (bal && ism) {
          int src = __ffs(bal) - 1;
          bal &= bal - 1;
          int ww = __shfl_sync(kFull, w, src);
          bool trivially = false;
          for (int q = 0; q < k - 1; ++q) trivially |= (t.v[q] == ww);
          if (trivially) continue;
          const int32_t* rw = g.col + g.row_off[ww];
          int dw = g.row_off[ww + 1] - g.row_off[ww];
          // ww covers L_parent only if it has at least |L_parent| neighbours;
          // otherwise it is a new R vertex below `last`: not maximal here.
          if (dw < nLp) {
            ism = false;
            break;
          }
          bool all = true;
          for (int j0 = 0; j0 < nLp && all; j0 += 32) {
            int j = j0 + lane;
            bool in = j >= nLp || contains_sorted(rw, dw, Lpar[j]);
            all = __all_sync(kFull, in);
          }
          if (!all) ism = false;
        }
      }
    }
  }
  if (!ism) {
    W.nonmax += 1;
    for (int i = lane; i < nt; i += 32) map[touched[i]] = 0;
    __syncwarp();
    return;
  }
  // the task's own biclique (once: parts after the first skip it)
  if (part == 0) {
    uint64_t sL = 0;
    for (int l = lane; l < nL; l += 32) sL += g.ukey[L[l]];
    sL = warp_sum(sL);
    W.cnt += 1;
    W.hash += biclique_hash(g, sL, (uint64_t)nL, sR, nR);
    if (W.p.emit) emit_list(W.ctl, emit_dst(W.p), W.gid, nL, L, nullptr);
  }
  bool done = nL <= 1 || np == 0;
  // ---- split (src/IterFinderGpu.cu:835-858) ----
  // A heavy root splits the same way in the sub-problem sharing mode: its
  // first level alone would otherwise run on one warp for the whole launch.
  if (!done && k < 4) {
    long long rest = np;
    bool split;
    if (W.p.vertex_split)
      split = (rest > W.gp->bound_height || nL > W.gp->bound_height) &&
              rest * (long long)nL > (long long)W.gp->bound_size;
    else
      split = k == 1 && parts <= 1 && W.p.root_split > 0 &&
              rest * (long long)nL > (long long)W.p.root_split;
    if (split) {
      if (queue_push_children(W, t, k, nq, nC)) {
        W.splits += 1;
        done = true;
      }
    }
  }
  if (!done) {
    if (nL <= W.gp->tier2_max_l && nC <= W.gp->direct_max_c) {
      // ---- tier 2 directly: masks of every candidate over all of L ----
      uint64_t* lkey = W.A64(W.sl.lkey);
      uint64_t* subkey = W.A64(W.sl.sub_v);
      int32_t* lid = W.A(W.sl.lid);
      for (int l = lane; l < nL; l += 32) lkey[l] = g.ukey[L[l]];
      if (W.p.emit)
        for (int l = lane; l < nL; l += 32) lid[l] = L[l];
      for (int i = lane; i < nC; i += 32) subkey[i] = g.vkey[cv[i]];
      const int K = words_k(nL), RS = rec_stride(K);
      uint32_t* rec = reinterpret_cast<uint32_t*>(W.A(W.sl.masks));
      init_records(rec, K, nC);
      flat_rows(
          nL,
          [&](int r, int& beg, int& len) {
            int u = L[r];
            beg = g.rev_off[u];
            len = g.rev_off[u + 1] - beg;
          },
          [&](bool valid, int r, int pos) {
            if (!valid) return;
            int p = map[__ldg(g.rev_col + pos)] - 1;
            if (p >= 0) atomicOr(&rec[(size_t)p * RS + 1 + (r >> 5)], 1u << (r & 31));
          });
      __syncwarp();
      tier2(W, nL, nC, nq, nend, sR, nR);
    } else {
      // ---- tier 1: local adjacency ----
      {
        uint64_t* ckey = W.A64(W.sl.ckey);  // hash key per candidate, for the pushes
        for (int i = lane; i < nC; i += 32) ckey[i] = g.vkey[cv[i]];
      }
      int32_t* llevel = W.A(W.sl.llevel);
      int32_t* aadj = W.A(W.sl.aadj);
      int32_t* coff = W.A(W.sl.coff);
      int32_t* fill = W.A(W.sl.fill);
      int32_t* cadj = W.A(W.sl.cadj);
      int32_t* sidx = W.A(W.sl.sidx);
      int32_t* ent = W.A(W.sl.ent);  // free until the first sparse push
      for (int l = lane; l < nL; l += 32) llevel[l] = 0;
      // aadj: L row -> C index (or -1 for R), rows sized by degree
      flat_rows(
          nL,
          [&](int r, int& beg, int& len) {
            int u = L[r];
            beg = g.rev_off[u];
            len = g.rev_off[u + 1] - beg;
          },
          [&](bool valid, int r, int pos) {
            if (!valid) return;
            int u = L[r];
            int off = aoff[r] + (pos - g.rev_off[u]);
            aadj[off] = map[__ldg(g.rev_col + pos)] - 1;
            ent[off] = r;  // the entry's row, for the transpose below
          });
      // coff = exclusive scan of the initial counts; fill = 0; sidx = -1
      {
        int run = 0;
        for (int c0 = 0; c0 < nC; c0 += 32) {
          int i = c0 + lane;
          int c = i < nC ? ncnt[i] : 0;
          int tot;
          int ex = warp_excl_scan(c, &tot);
          if (i < nC) {
            coff[i] = run + ex;
            fill[i] = 0;
            sidx[i] = -1;
          }
          run += tot;
        }
        if (lane == 0) coff[nC] = run;
      }
      __syncwarp();
      // cadj: C index -> L positions.  A linear pass over the entries: each
      // lane has four slot reservations in flight before it uses any.
      {
        const int S = aoff[nL];
        for (int j0 = 0; j0 < S; j0 += 128) {
          int pp[4], rr[4], ss[4];
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const int j = j0 + k * 32 + lane;
            pp[k] = j < S ? aadj[j] : -1;
            rr[k] = j < S ? ent[j] : 0;
          }
#pragma unroll
          for (int k = 0; k < 4; ++k) ss[k] = pp[k] >= 0 ? atomicAdd(&fill[pp[k]], 1) : 0;
#pragma unroll
          for (int k = 0; k < 4; ++k)
            if (pp[k] >= 0) cadj[coff[pp[k]] + ss[k]] = rr[k];
        }
      }
      __syncwarp();
      // fill doubles as the sparse push's child-count array: back to zero.
      for (int i = lane; i < nC; i += 32) fill[i] = 0;
      __syncwarp();
      T1 t1;
      t1.L = L;
      t1.nL = nL;
      t1.nC = nC;
      t1.nq = nq;
      t1.nend = nend;
      t1.sRtask = sR;
      t1.nRtask = nR;
      uint64_t t1s = globaltimer_ns();
      uint64_t t2_before = W.ns_t2;
      tier1_run(W, t1);
      W.ns_t1 += (globaltimer_ns() - t1s) - (W.ns_t2 - t2_before);
    }
  }
  __syncwarp();
  for (int i = lane; i < nt; i += 32) map[touched[i]] = 0;
  __syncwarp();
}

}  // namespace

// ---------------------------------------------------------------------------
// Maps a global root position to (graph, root vertex): positions are the
// graphs' root lists laid end to end (root_prefix[i] = roots before graph i).
__device__ __forceinline__ int graph_of_position(const long long* prefix, int n, long long pos) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (prefix[mid] <= pos) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Serving: claims a root of the oldest published graph that has roots left
// (lane 0).  Graphs are drained in publication order; a warp that finds the
// head graph exhausted moves the head on.  As for a static launch, the
// launch-wide pending count is raised before a claim but only while some
// published graph may have roots left: idle warps polling an empty arrival
// ring must leave it at zero, or the launch could never see itself quiet.
// A warp that saw the head below the tail just before another moved it past
// its graph claims nothing (that graph was exhausted), so the quiet test
// (pending == 0, head >= tail) loses no root.
__device__ bool serve_claim_root(Warp& W, Task* t) {
  const ServeLink& L = W.p.serve;
  volatile ServeCtl* sc = L.sctl;
  if (sc->arr_head >= sc->arr_tail) return false;
  // A launch that is ending takes no new roots: the host relaunches for them.
  if (*(volatile int32_t*)&W.ctl->closing) return false;
  atomicAdd(&W.ctl->pending, 1ULL);
  for (int tries = 0; tries < 64; ++tries) {
    const unsigned long long h = sc->arr_head;
    if (h >= sc->arr_tail) break;
    const uint32_t blk = *(volatile const uint32_t*)&L.arr_blk[h % (unsigned long long)L.arr_cap];
    ServeGraph* sg = serve_graph(W, (int32_t)blk);
    const unsigned long long r = atomicAdd(&sg->next_root, 1ULL);
    const DevGraph& g = sg->g;
    if (r < (unsigned long long)g.n_roots) {
      t->v[0] = g.root_end - 1 - (g.root_offset + (int)r * g.root_stride);
      t->v[1] = t->v[2] = t->v[3] = -1;
      t->graph = (int32_t)blk;
      t->part = t->parts = t->pad = 0;
      return true;
    }
    atomicCAS((unsigned long long*)&L.sctl->arr_head, h, h + 1);
  }
  atomicAdd(&W.ctl->pending, (unsigned long long)-1LL);
  return false;
}

// Serving: one task of graph `gid` finished (lane 0, after its results were
// added).  The task that brings the graph's pending count to zero writes the
// graph's completion record for the host.
__device__ void serve_task_done(Warp& W, int32_t gid) {
  const ServeLink& L = W.p.serve;
  ServeGraph* sg = serve_graph(W, gid);
  if (atomicAdd(&sg->pending, (unsigned long long)-1LL) != 1ULL) return;
  __threadfence();
  volatile ServeGraph* vs = sg;
  const unsigned long long c = vs->res[0], h = vs->res[1], nm = vs->res[2], req = vs->request;
  const unsigned long long pos = atomicAdd(&L.sctl->done_pos, 1ULL);
  volatile ServeDone* d = L.done + (pos % (unsigned long long)L.done_cap);
  d->request = req;
  d->count = c;
  d->hash = h;
  d->non_maximal = nm;
  // Every task of the graph reserved its records before it finished, so the
  // reservation counter now lies past all of them.
  d->emit_end = *(volatile unsigned long long*)&W.ctl->emit_pos;
  __threadfence_system();
  d->seq = pos + 1;
}

// The persistent loop.  kTiers: the launch has a big tier (p.n_big_warps >
// 0); without it every warp uses `sl` and the tier code compiles away.
template <bool kTiers>
__device__ __forceinline__ void enum_main(const DevGraph* graphs, const long long* root_prefix,
                                          unsigned long long* gres, const EnumParams& p,
                                          const ScratchLayout& sl, EnumCtl* ctl, Task* q_tasks,
                                          unsigned long long* q_seq, const SlotPool& pool,
                                          int32_t* scratch, unsigned long long* exit_ns) {
  uint64_t t_start = globaltimer_ns();
  const int lane = (int)lane_id();
  const int warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  // Two tiers: the first n_big_warps warps hold the big layout, then the
  // launch's layout follows for every other warp.
  const bool big = kTiers && warp_global < p.n_big_warps;
  Warp W{p, (kTiers && big) ? p.big_sl : sl};
  W.ctl = ctl;
  W.q_tasks = q_tasks;
  W.q_seq = q_seq;
  W.slots = pool.slots;
  W.bigslots = pool.big;
  W.big_bits = pool.big_bits;
  W.nbig = pool.nbig;
  W.import_cap = pool.import_cap;
  W.import_l = pool.import_l;
  W.import_s = pool.import_s;
  W.slot_bits = pool.bits;
  W.nslot = pool.nslot;
  if (!kTiers)
    W.base = scratch + (size_t)warp_global * (size_t)sl.words_per_warp;
  else
    W.base = big ? scratch + (size_t)warp_global * (size_t)p.big_sl.words_per_warp
                 : scratch + (size_t)p.n_big_warps * (size_t)p.big_sl.words_per_warp +
                       (size_t)(warp_global - p.n_big_warps) * (size_t)sl.words_per_warp;
  extern __shared__ uint32_t enum_smem[];
  W.seen = sl.seen_words && p.touch_scan <= 0
               ? enum_smem + (size_t)(threadIdx.x >> 5) * sl.seen_words
               : nullptr;
  W.gseen = reinterpret_cast<uint32_t*>(W.base + W.sl.gseen);
  if (W.seen) {
    for (int i = lane; i < sl.seen_words; i += 32) W.seen[i] = 0u;
    __syncwarp();
  }
  W.graphs = graphs;
  W.gp = graphs;
  W.gid = 0;
  W.cnt = W.hash = W.nonmax = W.splits = 0;
  W.ns_t1 = W.ns_t2 = W.n_t2 = 0;
  W.pushes = W.shape = 0;
  W.deadline = p.time_limit_ns > 0 ? t_start + (uint64_t)p.time_limit_ns : 0;
  W.dem = 0;
  W.dem_t = -(1LL << 62);
  uint64_t ns_idle = 0, n_tasks = 0, max_task = 0, max_info = 0, max_split = 0;
  uint64_t max_pushes = 0, max_shape = 0;
  int32_t max_gid = 0;
  const long long nroots = p.server ? 0 : root_prefix[p.n_graphs];
  uint64_t idle_since = 0;
  uint64_t busy_ns = 0, last_done_ns = 0, idle_last = 0;
  while (true) {
    int ab = 0;
    if (lane == 0 && p.server) ab = *(volatile int32_t*)&p.serve.sctl->stop;  // shutting down
    if (__shfl_sync(kFull, ab, 0) || must_stop(W)) break;
    Task t;
    int have = 0;
    if (lane == 0) {
      have = queue_pop(W, &t) ? 1 : 0;
      if (!have && p.server) {
        have = serve_claim_root(W, &t) ? 1 : 0;
      } else if (!have) {
        // A big warp first takes parts of big roots, then the roots no other
        // warp has room for.
        if (kTiers && big && p.big_parts_cap > 0) have = big_parts_claim(W, &t) ? 1 : 0;
        if (!have && kTiers && big &&
            *(volatile long long*)&ctl->next_big < (long long)p.n_big_roots) {
          atomicAdd(&ctl->pending, 1ULL);
          long long b = (long long)atomicAdd((unsigned long long*)&ctl->next_big, 1ULL);
          if (b < (long long)p.n_big_roots) {
            t.v[0] = p.big_roots[b];
            t.v[1] = t.v[2] = t.v[3] = -1;
            t.graph = 0;
            t.part = t.parts = t.pad = 0;
            have = 1;
          } else {
            atomicAdd(&ctl->pending, (unsigned long long)-1LL);
          }
        }
        if (!have && *(volatile long long*)&ctl->next_root < nroots) {
          atomicAdd(&ctl->pending, 1ULL);
          // Claims positions until one is not a listed big root (at most
          // every remaining position).
          while (true) {
            long long r = (long long)atomicAdd((unsigned long long*)&ctl->next_root, 1ULL);
            if (r >= nroots) {
              atomicAdd(&ctl->pending, (unsigned long long)-1LL);
              break;
            }
            int gi = graph_of_position(root_prefix, p.n_graphs, r);
            const DevGraph& gg = graphs[gi];
            long long k = r - root_prefix[gi];
            const int v = gg.root_end - 1 - (int)(gg.root_offset + k * gg.root_stride);
            if (kTiers && p.big_flag[v]) continue;
            t.v[0] = v;
            t.v[1] = t.v[2] = t.v[3] = -1;
            t.graph = gi;
            t.part = t.parts = t.pad = 0;
            have = 1;
            break;
          }
        }
      }
    }
    have = __shfl_sync(kFull, have, 0);
    if (have) {
#pragma unroll
      for (int i = 0; i < 4; ++i) t.v[i] = __shfl_sync(kFull, t.v[i], 0);
      t.graph = __shfl_sync(kFull, t.graph, 0);
      t.part = __shfl_sync(kFull, t.part, 0);
      t.parts = __shfl_sync(kFull, t.parts, 0);
      if (idle_since != 0 && lane == 0) atomicSub(&ctl->idle_warps, 1);
      uint64_t tb = globaltimer_ns();
      const unsigned long long t1_before = W.ns_t1, t2_before = W.ns_t2;
      const unsigned long long pushes_before = W.pushes;
      if (t.v[0] >= 0) {
        W.gid = t.graph;
        W.gp = graph_at(W, t.graph);
        run_task(W, t);
      } else if (t.v[1] == 1) {
        tier1_from_slot(W, -2 - t.v[0]);  // an exported counts-tier child (sets the graph)
      } else {
        tier2_from_slot(W, -2 - t.v[0]);  // an exported bitmap sub-problem (sets the graph)
      }
      __syncwarp();
      // Results go to the task's graph.
      if (lane == 0) {
        unsigned long long* r = p.server ? serve_graph(W, W.gid)->res : gres + 3 * (size_t)W.gid;
        if (W.cnt) atomicAdd(&r[0], W.cnt);
        if (W.hash) atomicAdd(&r[1], W.hash);
        if (W.nonmax) atomicAdd(&r[2], W.nonmax);
      }
      W.cnt = W.hash = W.nonmax = 0;
      uint64_t te = globaltimer_ns();
      busy_ns += te - tb;
      last_done_ns = te - t_start;
      ++n_tasks;
      if (te - tb > max_task) {
        max_task = te - tb;
        int nl = t.v[0] >= 0 ? W.gp->row_off[t.v[0] + 1] - W.gp->row_off[t.v[0]] : 0;
        max_info = ((unsigned long long)(unsigned)t.v[0] << 32) | (unsigned)nl;
        max_split = (W.ns_t1 - t1_before) / 1000 | ((W.ns_t2 - t2_before) / 1000 << 32);
        max_pushes = W.pushes - pushes_before;
        max_shape = t.v[0] >= 0 ? W.shape : 0;
        max_gid = W.gid;
      }
      if (lane == 0) {
        __threadfence();
        if (p.server) serve_task_done(W, W.gid);
        atomicAdd(&ctl->pending, (unsigned long long)-1LL);
      }
      idle_since = 0;
      continue;
    }
    // 1: leave now; 2 (serving): nothing in flight and no published roots left.
    // A serving launch ends as a whole: the first warp to see it quiet for
    // idle_exit_ns sets `closing`, after which no warp claims a new root and
    // every warp leaves once nothing is pending.  Graphs published meanwhile
    // wait for the host's next launch, which gets the whole grid.  (Warps
    // that left one by one would let arrivals keep a launch of a few
    // remaining warps alive indefinitely.)
    int finished = 0;
    if (lane == 0) {
      if (p.server) {
        volatile ServeCtl* sc = p.serve.sctl;
        const bool quiet = *(volatile unsigned long long*)&ctl->pending == 0ULL;
        if (sc->stop || (quiet && *(volatile int32_t*)&ctl->closing)) finished = 1;
        else if (quiet && sc->arr_head >= sc->arr_tail)
          finished = 2;
      } else {
        finished = (*(volatile long long*)&ctl->next_root >= nroots &&
                    (!kTiers ||
                     *(volatile long long*)&ctl->next_big >= (long long)p.n_big_roots) &&
                    *(volatile unsigned long long*)&ctl->pending == 0ULL)
                       ? 1
                       : 0;
      }
    }
    finished = __shfl_sync(kFull, finished, 0);
    if (finished == 1) break;
    uint64_t now = globaltimer_ns();
    if (idle_since != 0) ns_idle += now - idle_last;
    idle_last = now;
    if (idle_since == 0) {
      idle_since = now;
      if (lane == 0) atomicAdd(&ctl->idle_warps, 1);
    } else if (p.server && finished == 2 && now - idle_since > (uint64_t)p.serve.idle_exit_ns) {
      // A serving launch ends once it has had nothing to do for a while; the
      // host launches again when graphs arrive.
      if (lane == 0) {
        atomicExch(&ctl->closing, 1);
        atomicSub(&ctl->idle_warps, 1);
      }
      break;
    } else if (now - idle_since > (uint64_t)p.idle_ns_limit) {
      if (lane == 0) set_status(ctl, kStTimeout, now - idle_since);
      break;
    }
    __nanosleep(256);
  }
  __syncwarp();
  if (lane == 0) {
    if (W.splits) atomicAdd(&ctl->tasks_split, W.splits);
    atomicAdd(&ctl->ns_setup, (unsigned long long)(busy_ns - W.ns_t1 - W.ns_t2));
    atomicAdd(&ctl->ns_tier1, (unsigned long long)W.ns_t1);
    atomicAdd(&ctl->ns_tier2, (unsigned long long)W.ns_t2);
    atomicAdd(&ctl->ns_idle, (unsigned long long)ns_idle);
    atomicAdd(&ctl->n_tasks, (unsigned long long)n_tasks);
    atomicAdd(&ctl->n_tier2, (unsigned long long)W.n_t2);
    unsigned long long old = atomicMax(&ctl->max_task_ns, (unsigned long long)max_task);
    if (old < max_task) {
      atomicExch(&ctl->max_task_info, (unsigned long long)max_info);
      // (counts-tier us) | (bitmap-tier us << 32), and the task's graph
      atomicExch(&ctl->max_task_split, (unsigned long long)max_split);
      atomicExch(&ctl->max_task_graph, (unsigned long long)max_gid);
      atomicExch(&ctl->max_task_pushes, (unsigned long long)max_pushes);
      atomicExch(&ctl->max_task_shape, (unsigned long long)max_shape);
    }
  }
  if (p.record_exit) {
    // Per block: when its last task finished, and its warps' summed busy time.
    __shared__ unsigned long long blk_last, blk_busy;
    if (threadIdx.x == 0) {
      blk_last = 0;
      blk_busy = 0;
    }
    __syncthreads();
    if (lane == 0) {
      atomicMax(&blk_last, (unsigned long long)last_done_ns);
      atomicAdd(&blk_busy, (unsigned long long)busy_ns);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      exit_ns[blockIdx.x] = blk_last;
      exit_ns[gridDim.x + blockIdx.x] = blk_busy;
    }
  }
}

__global__ void __launch_bounds__(kEnumThreads, kEnumMinBlocks)
    mbe_enum_kernel(const DevGraph* graphs, const long long* root_prefix,
                    unsigned long long* gres, const __grid_constant__ EnumParams p,
                    const __grid_constant__ ScratchLayout sl, EnumCtl* ctl, Task* q_tasks,
                    unsigned long long* q_seq, SlotPool pool, int32_t* scratch,
                    unsigned long long* exit_ns) {
  enum_main<false>(graphs, root_prefix, gres, p, sl, ctl, q_tasks, q_seq, pool, scratch, exit_ns);
}

__global__ void __launch_bounds__(kEnumThreads, kEnumMinBlocks)
    mbe_enum_kernel_tiers(const DevGraph* graphs, const long long* root_prefix,
                          unsigned long long* gres, const __grid_constant__ EnumParams p,
                          const __grid_constant__ ScratchLayout sl, EnumCtl* ctl, Task* q_tasks,
                          unsigned long long* q_seq, SlotPool pool, int32_t* scratch,
                          unsigned long long* exit_ns) {
  enum_main<true>(graphs, root_prefix, gres, p, sl, ctl, q_tasks, q_seq, pool, scratch, exit_ns);
}

}  // namespace gmbe
