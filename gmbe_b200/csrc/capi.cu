// extern "C" layer: graph lifetime, device upload and the enumeration launch.
// See include/mbe.h for the contract and the reference interfaces replaced.
#include <cuda_runtime.h>
#include <sys/time.h>

#include <algorithm>
#include <iterator>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <chrono>
#include <functional>
#include <thread>

#include "engine.h"
#include "tiers.h"

using namespace gmbe;


namespace {

double now_s() {
  struct timeval tv;
  gettimeofday(&tv, nullptr);
  return (double)tv.tv_sec + (double)tv.tv_usec * 1e-6;
}

int cuda_fail(cudaError_t e, const char* what) {
  return set_error(MBE_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(call)                                        \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

inline uint64_t fmix64_h(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ULL;
  k ^= k >> 33;
  return k;
}

void free_device(mbe_graph* g) {
  cudaFree(g->d_row_off);
  cudaFree(g->d_col);
  cudaFree(g->d_rev_off);
  cudaFree(g->d_rev_col);
  cudaFree(g->d_ukey);
  cudaFree(g->d_vkey);
  g->d_row_off = g->d_col = g->d_rev_off = g->d_rev_col = nullptr;
  g->d_ukey = g->d_vkey = nullptr;
}

constexpr int kMaxDevices = 64;
Workspace g_ws[kMaxDevices];

template <typename T>
int upload(T** dst, const std::vector<T>& src) {
  size_t n = std::max<size_t>(src.size(), 1);
  CK(cudaMalloc((void**)dst, n * sizeof(T)));
  if (!src.empty()) CK(cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
  return MBE_OK;
}

int upload_graph(mbe_graph* g) {
  CK(cudaSetDevice(g->device));
  const HostGraph& h = g->h;
  int rc;
  if ((rc = upload(&g->d_row_off, h.row_off))) return rc;
  if ((rc = upload(&g->d_col, h.col))) return rc;
  if ((rc = upload(&g->d_rev_off, h.rev_off))) return rc;
  if ((rc = upload(&g->d_rev_col, h.rev_col))) return rc;
  std::vector<uint64_t> uk, vk;
  host_keys(h, &uk, &vk);
  if ((rc = upload(&g->d_ukey, uk))) return rc;
  if ((rc = upload(&g->d_vkey, vk))) return rc;
  return graph_caps(h, &g->capL, &g->capS);
}

int finish_graph(mbe_graph* g, mbe_graph** out) {
  int rc = upload_graph(g);
  if (rc) {
    free_device(g);
    delete g;
    return rc;
  }
  *out = g;
  return MBE_OK;
}

}  // namespace

namespace gmbe {

Workspace& workspace(int device) { return g_ws[device]; }

void host_keys(const HostGraph& h, std::vector<uint64_t>* uk, std::vector<uint64_t>* vk) {
  // Keys in original ids and original sides (see include/mbe.h).
  uk->resize(h.U_size);
  vk->resize(h.V_size);
  for (int32_t u = 0; u < h.U_size; ++u)
    (*uk)[u] = fmix64_h((uint64_t)h.u_orig[u] * 2u + (h.swapped ? 1u : 0u));
  for (int32_t v = 0; v < h.V_size; ++v)
    (*vk)[v] = fmix64_h((uint64_t)h.v_orig[v] * 2u + (h.swapped ? 0u : 1u));
}

int graph_caps(const HostGraph& h, int32_t* capL_out, int32_t* capS_out) {
  int64_t capS = 0;
  int32_t capL = 0;
  for (int32_t v = 0; v < h.V_size; ++v) {
    int64_t s = 0;
    for (int32_t i = h.row_off[v]; i < h.row_off[v + 1]; ++i) {
      int32_t u = h.col[i];
      s += h.rev_off[u + 1] - h.rev_off[u];
    }
    capS = std::max(capS, s);
    capL = std::max(capL, h.row_off[v + 1] - h.row_off[v]);
  }
  if (capS > INT32_MAX / 2)
    return set_error(MBE_ERR_CAPACITY, "two-hop multiset of a root exceeds 2^30 entries");
  *capS_out = (int32_t)std::max<int64_t>(capS, 1);
  *capL_out = std::max(capL, 1);
  return MBE_OK;
}

ScratchLayout make_layout(int32_t nV, int32_t capC, int32_t capL, int32_t capS) {
  ScratchLayout s;
  memset(&s, 0, sizeof(s));
  s.capC = capC;
  s.capL = capL;
  s.capS = capS;
  s.kmax = kKMax;
  int64_t off = 0;
  auto take = [&](int64_t words) {
    int64_t o = off;
    off += (words + 7) & ~int64_t(7);  // 32-byte aligned slices
    return o;
  };
  const int64_t C = capC, Lc = capL, S = capS, T2 = 32 * kKMax;
  s.map = take(nV);
  s.gseen_words = (int32_t)((std::max<int64_t>(nV, C) + 31) / 32);
  s.gseen = take(s.gseen_words);
  s.zero_words = off;
  s.touched = take(C);
  s.cv = take(C);
  s.ncnt = take(C);
  s.bound = take(C);
  s.coff = take(C + 1);
  s.fill = take(C);
  s.sidx = take(C);
  s.lv = take(Lc);
  s.llevel = take(Lc);
  s.lp = take(Lc);
  s.aoff = take(Lc + 1);
  s.stack = take(Lc + 2);
  s.lent = take(Lc + 2);
  s.lbits = take((int64_t)kLevelBits * ((C + 31) / 32));
  s.aadj = take(S);
  s.cadj = take(S);
  s.masks = take((int64_t)(kKMax + 1) * C);  // bitmap-tier records (K+1 words each)
  s.sub_v = take(2 * C);
  s.tcls = take(C);
  s.ckey = take(2 * C);
  s.ent = take(S);
  s.lkey = take(2 * T2);
  s.lid = take(T2);
  s.lmask = take((T2 + 3) * kKMax);
  s.t2_rec = take(2 * (T2 + 3));
  s.t2_n = take(T2 + 3);
  s.t2_cur = take(T2 + 3);
  s.t2_top = take(T2 + 3);
  s.r_sum = take(2 * (T2 + 3));
  s.r_cnt = take(T2 + 3);
  s.tlist = take(C);
  // Arena of the bitmap tier's per-level record lists (a level that does not
  // fit shares its parent's list).
  s.act_cap = (int32_t)std::min<int64_t>(INT32_MAX / 2, 6 * C + 8192);
  s.act = take(s.act_cap);
  s.words_per_warp = off;
  const int64_t seen = ((int64_t)nV + 31) / 32;
  s.seen_words = seen <= kSeenMaxWords ? (int32_t)seen : 0;
  return s;
}

int choose_tiers(int32_t nV, int32_t n_roots, const int64_t* S, const int32_t* D,
                 const int32_t* roots, int warps, uint64_t budget, int64_t force_bound,
                 int32_t force_big, TierChoice* out, std::vector<int32_t>* list,
                 std::vector<uint8_t>* flags, bool pool_for_parts) {
  *out = TierChoice();
  list->clear();
  flags->clear();
  nV = std::max<int32_t>(nV, 1);
  auto bytes_of = [&](const TierCaps& c) {
    return (uint64_t)make_layout(nV, c.capC, c.capL, c.capS).words_per_warp * sizeof(int32_t);
  };
  // The launch's own capacities: tasks below a root (its children and
  // exported sub-problems) never need more than the root.
  TierCaps full;
  int64_t s_max = 1;
  for (int32_t k = 0; k < n_roots; ++k) {
    s_max = std::max(s_max, S[k]);
    full.capL = std::max(full.capL, D[k]);
  }
  if (s_max > INT32_MAX / 2)
    return set_error(MBE_ERR_CAPACITY, "two-hop multiset of a root exceeds 2^30 entries");
  full.capS = (int32_t)s_max;
  full.capC = std::max<int32_t>(1, std::min<int32_t>(nV, full.capS));
  const uint64_t full_b = bytes_of(full);
  out->small = out->big = full;
  out->small_bytes = out->big_bytes = full_b;
  if (force_bound <= 0 && full_b * (uint64_t)warps <= budget) return MBE_OK;

  // The small tier must hold any exported sub-problem a big warp makes.
  const int32_t min_c = std::min<int32_t>(full.capC, kSlotMaxRecords);
  auto small_caps = [&](int64_t T) {
    TierCaps c;
    for (int32_t k = 0; k < n_roots; ++k)
      if (S[k] <= T) c.capL = std::max(c.capL, D[k]);
    c.capS = (int32_t)std::max<int64_t>(1, std::min<int64_t>(T, full.capS));
    c.capC = std::max(min_c, std::max<int32_t>(1, std::min<int32_t>(nV, c.capS)));
    c.capL = std::min(c.capL, full.capL);
    return c;
  };
  int64_t T = force_bound;
  if (T <= 0) {
    T = (int64_t)1 << 16;
    for (int64_t t = T; t < full.capS; t <<= 1)
      if (bytes_of(small_caps(t)) * (uint64_t)warps <= budget / 10 * 6) T = t;
  }
  flags->assign((size_t)nV, 0);
  for (int32_t k = 0; k < n_roots; ++k)
    if (S[k] > T) {
      list->push_back(roots[k]);
      (*flags)[(size_t)roots[k]] = 1;
    }
  if (list->empty()) {  // every root fits the bound: one tier, if it fits at all
    flags->clear();
    if (force_bound <= 0 && full_b * (uint64_t)warps > budget)
      return set_error(MBE_ERR_NOMEM,
                       "scratch of %d warps: %.2f GB of %.2f GB, and no root is above the "
                       "two-hop bound %lld that a second tier would take",
                       warps, full_b * (double)warps / 1e9, budget / 1e9, (long long)T);
    return MBE_OK;
  }
  const TierCaps small = small_caps(T);
  const uint64_t small_b = bytes_of(small);
  if (small_b * (uint64_t)warps > budget)
    return set_error(MBE_ERR_NOMEM, "scratch of %d warps at two-hop bound %lld: %.2f GB of %.2f GB",
                     warps, (long long)T, small_b * (double)warps / 1e9, budget / 1e9);
  const uint64_t extra = full_b > small_b ? full_b - small_b : 0;
  const int64_t fit = extra ? (int64_t)((budget - small_b * (uint64_t)warps) / extra) : warps;
  const int64_t want = pool_for_parts ? (int64_t)warps : (int64_t)list->size();
  int64_t n_big = force_big > 0 ? force_big
                                : std::min<int64_t>({want, fit, (int64_t)warps / 2});
  n_big = std::min<int64_t>(n_big, warps);
  if (n_big < 1 || n_big > fit)
    return set_error(MBE_ERR_NOMEM, "%lld warps for the largest roots (%.2f GB each) do not fit",
                     (long long)std::max<int64_t>(n_big, 1), full_b / 1e9);
  out->n_big = (int32_t)n_big;
  out->bound = T;
  out->small = small;
  out->small_bytes = small_b;
  return MBE_OK;
}


int apply_tuning(const mbe_params& prm, DevGraph* dg) {
  int t2 = prm.bitmap_max_l;
  if (t2 == 0) t2 = 32 * kKMax;
  if (t2 < 0) t2 = 1;
  if (t2 > 32 * kKMax) return set_error(MBE_ERR_INVALID, "bitmap_max_l > %d", 32 * kKMax);
  dg->bound_height = prm.bound_height;
  dg->bound_size = prm.bound_size;
  dg->tier2_max_l = t2;
  dg->direct_max_c = prm.direct_max_c > 0 ? prm.direct_max_c : 16384;
  return MBE_OK;
}

int enum_blocks_per_sm(bool tiers, size_t smem, int* occ) {
  const void* fn = tiers ? (const void*)mbe_enum_kernel_tiers : (const void*)mbe_enum_kernel;
  // The limit only ever rises: a server and single-graph launches may share
  // the kernel from different threads, each with its own bitmap size.
  cudaFuncAttributes fa;
  CK(cudaFuncGetAttributes(&fa, fn));
  if ((size_t)fa.maxDynamicSharedSizeBytes < smem)
    CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, fn, kEnumThreads, smem));
  if (*occ < 1) return set_error(MBE_ERR_CUDA, "enumeration kernel cannot be resident");
  return MBE_OK;
}

int engine_prepare(Workspace& ws, const LaunchSpec& spec, const mbe_params& prm, LaunchPlan* plan) {
  if (!ws.ev0) {
    CK(cudaEventCreate(&ws.ev0));
    CK(cudaEventCreate(&ws.ev1));
  }
  if (spec.capC >= (1 << 24))
    return set_error(MBE_ERR_CAPACITY, "candidate sets above 2^24 entries are not supported");
  plan->sl = make_layout(spec.map_words, spec.capC, spec.capL, spec.capS);
  int dev_sms = 0;
  CK(cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, spec.device));
  // Every block of the persistent launch is resident at once.
  int occ = 0;
  int rc = enum_blocks_per_sm(spec.n_big > 0, enum_smem_bytes(plan->sl), &occ);
  if (rc) return rc;
  plan->blocks = prm.blocks > 0 ? std::min(prm.blocks, dev_sms * occ) : dev_sms * occ;
  plan->warps = plan->blocks * kEnumWarps;
  // The big tier (if any): the first n_big warps.  Both layouts share the
  // count-map size, hence the shared-memory bitmap.
  const int n_big = std::max(0, std::min(spec.n_big, plan->warps));
  ScratchLayout big_sl;
  memset(&big_sl, 0, sizeof(big_sl));
  if (n_big > 0) {
    if (spec.bigC >= (1 << 24))
      return set_error(MBE_ERR_CAPACITY, "candidate sets above 2^24 entries are not supported");
    big_sl = make_layout(spec.map_words, spec.bigC, spec.bigL, spec.bigS);
  }
  plan->map_words = spec.map_words;
  size_t need = scratch_bytes(plan->sl, big_sl, plan->warps, n_big);
  if (need > ws.scratch_bytes) {
    cudaFree(ws.scratch);
    ws.scratch = nullptr;
    ws.scratch_bytes = 0;
    cudaError_t e = cudaMalloc((void**)&ws.scratch, need);
    if (e != cudaSuccess)
      return set_error(MBE_ERR_NOMEM, "scratch of %.2f GB: %s", need / 1e9, cudaGetErrorString(e));
    ws.scratch_bytes = need;
    ws.map_pitch_words = -1;
    ++ws.gen;
  }
  // Every task leaves its warp's dense count map all-zero.  A different
  // layout puts the maps elsewhere: they are cleared (strided, maps only).
  plan->clear_maps = ws.map_pitch_words != plan->sl.words_per_warp ||
                     ws.map_words != spec.map_words || ws.map_warps < plan->warps ||
                     ws.map_big != n_big || ws.map_big_pitch != big_sl.words_per_warp;
  int32_t qcap = prm.queue_capacity > 0
                     ? prm.queue_capacity
                     : (int32_t)std::min<int64_t>(1 << 22,
                                                  std::max<int64_t>(1 << 16, 8LL * spec.map_words));
  if (qcap != ws.q_cap) {
    cudaFree(ws.q_tasks);
    cudaFree(ws.q_seq);
    ws.q_tasks = nullptr;
    ws.q_seq = nullptr;
    ws.q_cap = 0;
    CK(cudaMalloc((void**)&ws.q_tasks, sizeof(Task) * (size_t)qcap));
    CK(cudaMalloc((void**)&ws.q_seq, sizeof(unsigned long long) * (size_t)qcap));
    ws.q_cap = qcap;
    ++ws.gen;
  }
  if (!ws.ctl) {
    CK(cudaMalloc((void**)&ws.ctl, sizeof(EnumCtl)));
    ++ws.gen;
  }
  if (!ws.slots) {
    const int32_t nslot = 4096;  // 4096 x 128 KiB = 512 MiB
    CK(cudaMalloc((void**)&ws.slots, sizeof(int32_t) * (size_t)kSlotWordsHost * nslot));
    CK(cudaMalloc((void**)&ws.slot_bits, sizeof(uint32_t) * (size_t)(nslot / 32)));
    ws.nslot = nslot;
    ++ws.gen;
  }
  if (!ws.big_slots) {
    // Large slots: children with more candidates than a regular slot holds
    // (graphs whose candidate sets reach hundreds of thousands) can still go
    // to idle warps.  128 x 4 MiB = 512 MiB.
    const int32_t nbig = 128;
    CK(cudaMalloc((void**)&ws.big_slots, sizeof(int32_t) * (size_t)kBigSlotWords * nbig));
    CK(cudaMalloc((void**)&ws.big_slot_bits, sizeof(uint32_t) * (size_t)(nbig / 32)));
    ws.nbig_slot = nbig;
    ++ws.gen;
  }
  if (plan->blocks > ws.exit_cap) {
    cudaFree(ws.exit_ns);
    ws.exit_ns = nullptr;
    ws.exit_cap = 0;
    CK(cudaMalloc((void**)&ws.exit_ns, 2 * sizeof(unsigned long long) * (size_t)plan->blocks));
    ws.exit_cap = plan->blocks;
    ++ws.gen;
  }
  if (!ws.d_graph1) {
    CK(cudaMalloc((void**)&ws.d_graph1, sizeof(DevGraph)));
    CK(cudaMalloc((void**)&ws.d_prefix1, 2 * sizeof(long long)));
    CK(cudaMalloc((void**)&ws.d_gres1, 3 * sizeof(unsigned long long)));
  }
  EnumParams& ep = plan->ep;
  memset(&ep, 0, sizeof(ep));
  ep.prune = prm.prune;
  ep.queue_cap = qcap;
  ep.slot_spin_limit = 20000000;  // x ~64 ns sleeps: a claimed slot is written within microseconds
  ep.idle_ns_limit = prm.wait_limit_ns > 0 ? prm.wait_limit_ns : 600LL * 1000000000LL;
  ep.time_limit_ns = std::max<int64_t>(prm.time_limit_ns, 0);
  ep.touch_scan = prm.touch_scan > 0 ? 1 : (prm.touch_scan < 0 ? -1 : 0);
  ep.slot_records = std::max(prm.slot_records, 0);
  ep.share_counts = prm.share_counts < 0 ? 0 : 1;
  ep.record_exit = prm.sm_timing ? 1 : 0;
  ep.vertex_split = prm.split_mode == 1 ? 1 : 0;
  // Heavy roots split into vertex tuples (sub-problem sharing mode only).
  ep.root_split = prm.split_mode == 1 ? 0 : std::max(prm.root_split_size, 0);
  ep.share_min_work = prm.share_min_work > 0 ? prm.share_min_work : kShareMinWorkDefault;
  apply_range_split(prm, &ep.range_work, &ep.range_chunk);
  // Heavy roots are split into parts by default: single roots with |P|*|C|
  // above 10^9 (graphs of hundreds of thousands of candidates per root)
  // otherwise run for most of a launch on one warp.
  if (prm.range_split_work == 0 && prm.split_mode != 1) ep.range_work = kRangeWorkDefault;
  ep.eager_share = eager_share_of(prm);
  ep.n_graphs = spec.n_graphs;
  ep.n_big_warps = n_big;
  ep.big_sl = big_sl;
  if (n_big > 0) {
    // Vertex-tuple children could need the big tier: off.  Root parts stay
    // on (a big root's parts run on big warps only).
    ep.root_split = 0;
  }
  plan->pool.slots = ws.slots;
  plan->pool.bits = ws.slot_bits;
  plan->pool.nslot = prm.split_mode == 1 ? 0 : ws.nslot;
  plan->pool.big = ws.big_slots;
  plan->pool.big_bits = ws.big_slot_bits;
  plan->pool.nbig = prm.split_mode == 1 ? 0 : ws.nbig_slot;
  // The small tier's capacities: every warp has at least these.
  plan->pool.import_cap = plan->sl.capC;
  plan->pool.import_l = plan->sl.capL;
  plan->pool.import_s = plan->sl.capS;
  plan->pool.pad = 0;
  return MBE_OK;
}

int engine_clear_maps(Workspace& ws, LaunchPlan* plan, cudaStream_t st) {
  if (!plan->clear_maps) return MBE_OK;
  // The count map and the global first-touch bitmap are the first slices of
  // either layout.
  const int n_big = plan->ep.n_big_warps;
  const size_t big_pitch = (size_t)plan->ep.big_sl.words_per_warp;
  if (n_big > 0)
    CK(cudaMemset2DAsync(ws.scratch, big_pitch * sizeof(int32_t), 0,
                         (size_t)plan->ep.big_sl.zero_words * sizeof(int32_t), (size_t)n_big, st));
  if (plan->warps > n_big)
    CK(cudaMemset2DAsync(ws.scratch + big_pitch * (size_t)n_big,
                         (size_t)plan->sl.words_per_warp * sizeof(int32_t), 0,
                         (size_t)plan->sl.zero_words * sizeof(int32_t),
                         (size_t)(plan->warps - n_big), st));
  ws.map_pitch_words = plan->sl.words_per_warp;
  ws.map_words = plan->map_words;
  ws.map_warps = plan->warps;
  ws.map_big = n_big;
  ws.map_big_pitch = (int64_t)big_pitch;
  plan->clear_maps = false;
  return MBE_OK;
}

int engine_enqueue(Workspace& ws, LaunchPlan* plan, const DevGraph* d_graphs,
                   const long long* d_prefix, unsigned long long* d_gres, int n_graphs,
                   cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1) {
  int rc = engine_clear_maps(ws, plan, st);
  if (rc) return rc;
  CK(cudaMemsetAsync(ws.ctl, 0, sizeof(EnumCtl), st));
  CK(cudaMemsetAsync(ws.q_seq, 0, sizeof(unsigned long long) * (size_t)ws.q_cap, st));
  CK(cudaMemsetAsync(ws.slot_bits, 0, sizeof(uint32_t) * (size_t)(ws.nslot / 32), st));
  CK(cudaMemsetAsync(ws.big_slot_bits, 0, sizeof(uint32_t) * (size_t)(ws.nbig_slot / 32), st));
  CK(cudaMemsetAsync(d_gres, 0, 3 * sizeof(unsigned long long) * (size_t)n_graphs, st));
  if (ev0) CK(cudaEventRecord(ev0, st));
  auto* kernel = plan->ep.n_big_warps > 0 ? mbe_enum_kernel_tiers : mbe_enum_kernel;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)plan->blocks);
  cfg.blockDim = dim3(kEnumThreads);
  cfg.dynamicSmemBytes = enum_smem_bytes(plan->sl);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  if (plan->l2_bytes > 0) {
    // The hot read-only data (the graph's U -> V lists, walked by every task
    // set-up) persists in L2 while the warps' scratch streams through it.
    attr[0].id = cudaLaunchAttributeAccessPolicyWindow;
    attr[0].val.accessPolicyWindow.base_ptr = const_cast<void*>(plan->l2_base);
    attr[0].val.accessPolicyWindow.num_bytes = plan->l2_bytes;
    attr[0].val.accessPolicyWindow.hitRatio = plan->l2_hit;
    attr[0].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    attr[0].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
  }
  CK(cudaLaunchKernelEx(&cfg, kernel, d_graphs, d_prefix, d_gres, plan->ep, plan->sl, ws.ctl,
                        ws.q_tasks, ws.q_seq, plan->pool, ws.scratch, ws.exit_ns));
  if (ev1) CK(cudaEventRecord(ev1, st));
  return MBE_OK;
}

int engine_status(Workspace& ws, const EnumCtl& ctl) {
  if (ctl.status == 0) return MBE_OK;
  // An aborted run leaves count maps dirty: clear them on the next call.
  ws.map_pitch_words = -1;
  switch (ctl.status) {
    case kStTimeout:
      return set_error(MBE_ERR_TIMEOUT, "device wait limit reached (idle %llu ns)", ctl.err_info);
    case kStQueue:
      return set_error(MBE_ERR_TIMEOUT, "split-queue slot %llu was never written", ctl.err_info);
    case kStCapacity:
      return set_error(MBE_ERR_CAPACITY, "scratch capacity exceeded (info 0x%llx)", ctl.err_info);
    case kStDeadline:
      return set_error(MBE_ERR_TIMEOUT, "launch time limit reached (result incomplete)");
    default:
      return set_error(MBE_ERR_CUDA, "device status %d", ctl.status);
  }
}

void fill_profile(const EnumCtl& ctl, mbe_result* out) {
  out->tasks_split = ctl.tasks_split;
  out->status = ctl.status;
  out->setup_ms = ctl.ns_setup / 1e6;
  out->tier1_ms = ctl.ns_tier1 / 1e6;
  out->tier2_ms = ctl.ns_tier2 / 1e6;
  out->idle_ms = ctl.ns_idle / 1e6;
  out->max_task_ms = ctl.max_task_ns / 1e6;
  out->max_task_root = (int32_t)(ctl.max_task_info >> 32);
  out->max_task_degree = (int32_t)(ctl.max_task_info & 0xffffffffu);
  out->max_task_tier1_ms = (double)(ctl.max_task_split & 0xffffffffu) / 1e3;
  out->max_task_tier2_ms = (double)(ctl.max_task_split >> 32) / 1e3;
  out->max_task_pushes1 = ctl.max_task_pushes & 0xffffffffu;
  out->max_task_pushes2 = ctl.max_task_pushes >> 32;
  out->max_task_cands = (int32_t)(ctl.max_task_shape & 0xffffffffu);
  out->max_task_part = (int32_t)((ctl.max_task_shape >> 32) & 0xffff);
  out->max_task_parts = (int32_t)(ctl.max_task_shape >> 48);
  out->max_task_graph = (int32_t)ctl.max_task_graph;
  out->n_tasks = ctl.n_tasks;
  out->n_subproblems = ctl.n_tier2;
}

}  // namespace gmbe

extern "C" {

void mbe_params_default(mbe_params* p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->bound_height = 20;
  p->bound_size = 1500;
  p->prune = 1;
}

void mbe_opts_default(mbe_opts* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->order = 1;  // reference Option() default (src/BiGraph.h:17-21)
}

int mbe_graph_from_csr(const int32_t* row_off, const int32_t* col, int32_t nV, int32_t nU,
                       int64_t nE, const mbe_opts* opts, mbe_graph** out) {
  clear_error();
  if (!out) return set_error(MBE_ERR_INVALID, "null output handle");
  *out = nullptr;
  mbe_opts o;
  if (opts) o = *opts;
  else mbe_opts_default(&o);
  if (o.device < 0 || o.device >= kMaxDevices) return set_error(MBE_ERR_INVALID, "bad device");
  mbe_graph* g = new mbe_graph();
  g->opts = o;
  g->device = o.device;
  int rc = build_host_graph(row_off, col, nV, nU, nE, o, &g->h);
  if (rc) {
    delete g;
    return rc;
  }
  return finish_graph(g, out);
}

int mbe_graph_build_on_device(const int32_t* row_off, const int32_t* col, int32_t nV, int32_t nU,
                              int64_t nE, const mbe_opts* opts, mbe_graph** out) {
  clear_error();
  if (!out) return set_error(MBE_ERR_INVALID, "null output handle");
  *out = nullptr;
  mbe_opts o;
  if (opts) o = *opts;
  else mbe_opts_default(&o);
  // The two-hop statistics (and the -o 3 peeling order they come with) are
  // host work: without fast_mode the graph is built as mbe_graph_from_csr does.
  if (!o.fast_mode) return mbe_graph_from_csr(row_off, col, nV, nU, nE, &o, out);
  if (o.device < 0 || o.device >= kMaxDevices) return set_error(MBE_ERR_INVALID, "bad device");
  mbe_graph* g = new mbe_graph();
  g->opts = o;
  g->device = o.device;
  int rc = device_build_graph(g, row_off, col, nV, nU, nE);
  if (rc) {
    free_device(g);
    delete g;
    return rc;
  }
  *out = g;
  return MBE_OK;
}

int mbe_graph_from_adj(const char* path, const mbe_opts* opts, mbe_graph** out) {
  clear_error();
  if (!path || !out) return set_error(MBE_ERR_INVALID, "null argument");
  *out = nullptr;
  std::vector<int32_t> ro, co;
  int32_t nU = 0;
  int rc = read_adj_file(path, &ro, &co, &nU);
  if (rc) return rc;
  return mbe_graph_from_csr(ro.data(), co.data(), (int32_t)ro.size() - 1, nU, (int64_t)co.size(),
                            opts, out);
}

int mbe_graph_get_info(const mbe_graph* g, mbe_graph_info* info) {
  clear_error();
  if (!g || !info) return set_error(MBE_ERR_INVALID, "null argument");
  info->U_size = g->h.U_size;
  info->V_size = g->h.V_size;
  info->edge_size = g->h.edge_size;
  info->U_degree = g->h.U_degree;
  info->V_degree = g->h.V_degree;
  info->U_2degree = g->h.U_2degree;
  info->V_2degree = g->h.V_2degree;
  info->swapped = g->h.swapped;
  return MBE_OK;
}

int mbe_device_release(int32_t device) {
  clear_error();
  if (device < 0 || device >= kMaxDevices) return set_error(MBE_ERR_INVALID, "bad device");
  Workspace& ws = g_ws[device];
  std::lock_guard<std::mutex> lock(ws.mu);
  CK(cudaSetDevice(device));
  CK(cudaDeviceSynchronize());
  for (void* p : {(void*)ws.scratch, (void*)ws.ctl, (void*)ws.q_tasks, (void*)ws.q_seq,
                  (void*)ws.exit_ns, (void*)ws.slots, (void*)ws.slot_bits, (void*)ws.big_slots,
                  (void*)ws.big_slot_bits, (void*)ws.d_graph1, (void*)ws.d_prefix1,
                  (void*)ws.d_gres1, (void*)ws.big_roots, (void*)ws.big_flag, (void*)ws.big_parts})
    cudaFree(p);
  ws.scratch = nullptr;
  ws.scratch_bytes = 0;
  ws.ctl = nullptr;
  ws.q_tasks = nullptr;
  ws.q_seq = nullptr;
  ws.q_cap = 0;
  ws.exit_ns = nullptr;
  ws.exit_cap = 0;
  ws.slots = nullptr;
  ws.slot_bits = nullptr;
  ws.nslot = 0;
  ws.big_slots = nullptr;
  ws.big_slot_bits = nullptr;
  ws.nbig_slot = 0;
  ws.d_graph1 = nullptr;
  ws.d_prefix1 = nullptr;
  ws.d_gres1 = nullptr;
  ws.big_roots = nullptr;
  ws.big_flag = nullptr;
  ws.big_parts = nullptr;
  ws.big_roots_cap = ws.big_flag_cap = ws.big_parts_cap = 0;
  ws.map_pitch_words = ws.map_words = -1;
  ws.map_warps = -1;
  ++ws.gen;  // captured batch launches refer to the old buffers
  return MBE_OK;
}

int mbe_graph_free(mbe_graph* g) {
  clear_error();
  if (!g) return MBE_OK;
  cudaSetDevice(g->device);
  free_device(g);
  delete g;
  return MBE_OK;
}


namespace {

// The scratch plan of one single-graph launch (see choose_tiers): the whole
// graph with the graph's capacities while one layout for every warp fits the
// device (no per-root pass); otherwise, and for explicit root ranges, sized
// from this launch's roots, in two tiers where one does not fit.
int plan_two_tiers(mbe_graph* g, const mbe_params& prm, int32_t rb, int32_t re, int32_t si,
                   int32_t sc, int32_t n_roots, size_t reusable_bytes, LaunchSpec* spec,
                   std::vector<int32_t>* list, std::vector<uint8_t>* flags) {
  const int32_t nV = std::max<int32_t>(g->h.V_size, 1);
  int dev_sms = 0, occ = 0;
  CK(cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, g->device));
  {
    const ScratchLayout whole = make_layout(nV, spec->capC, spec->capL, spec->capS);
    int rc = enum_blocks_per_sm(false, enum_smem_bytes(whole), &occ);
    if (rc) return rc;
  }
  const int blocks = prm.blocks > 0 ? std::min(prm.blocks, dev_sms * std::max(occ, 1))
                                    : dev_sms * std::max(occ, 1);
  const int warps = blocks * kEnumWarps;
  size_t free_b = 0, total_b = 0;
  CK(cudaMemGetInfo(&free_b, &total_b));
  // What the scratch may take: free memory plus the scratch the workspace
  // already holds, less room for the queue, slots and the caller's arrays.
  const size_t reserve = ((size_t)2 << 30) + total_b / 50;
  const size_t avail = free_b + reusable_bytes;
  const size_t budget = avail > reserve ? avail - reserve : 0;
  const size_t graph_b =
      (size_t)make_layout(nV, spec->capC, spec->capL, spec->capS).words_per_warp * sizeof(int32_t);
  const bool sub_range = rb > 0 || re < g->h.V_size;
  if (!sub_range && prm.big_two_hop <= 0 && graph_b * (size_t)warps <= budget) return MBE_OK;
  if (n_roots == 0) {  // nothing to enumerate: the smallest layout
    spec->capC = spec->capL = spec->capS = 1;
    return MBE_OK;
  }
  // Two-hop multiset and degree of every root of this launch.
  int rc = ensure_host_csr(g);
  if (rc) return rc;
  const HostGraph& h = g->h;
  std::vector<int64_t> S((size_t)n_roots);
  std::vector<int32_t> D((size_t)n_roots), roots((size_t)n_roots);
  for (int32_t k = 0; k < n_roots; ++k) {
    const int32_t v = re - 1 - (si + k * sc);
    int64_t s = 0;
    for (int32_t i = h.row_off[v]; i < h.row_off[v + 1]; ++i) {
      const int32_t u = h.col[i];
      s += h.rev_off[u + 1] - h.rev_off[u];
    }
    S[(size_t)k] = s;
    D[(size_t)k] = h.row_off[v + 1] - h.row_off[v];
    roots[(size_t)k] = v;
  }
  TierChoice ch;
  const bool parts = prm.split_mode != 1 && prm.range_split_work >= 0;
  if ((rc = choose_tiers(nV, n_roots, S.data(), D.data(), roots.data(), warps, budget,
                         prm.big_two_hop, prm.big_warps, &ch, list, flags, parts)))
    return rc;
  if (ch.n_big > 0 && prm.split_mode == 1)
    return set_error(MBE_ERR_INVALID, "split_mode 1 needs one scratch tier for every warp");
  spec->capC = ch.small.capC;
  spec->capL = ch.small.capL;
  spec->capS = ch.small.capS;
  spec->n_big = ch.n_big;
  spec->bigC = ch.big.capC;
  spec->bigL = ch.big.capL;
  spec->bigS = ch.big.capS;
  return MBE_OK;
}

}  // namespace

// mbe_enumerate, optionally writing biclique records into d_emit (emit_cap
// words) and reporting the words reserved in *emit_pos.  With d_emit_read
// (ring mode) the records go to a ring the host drains: `drain` runs in this
// thread, over and over, until the launch has finished.
static int enumerate_graph(mbe_graph* g, const mbe_params* params, mbe_result* out,
                           int32_t* d_emit, long long emit_cap, unsigned long long* emit_pos,
                           const unsigned long long* d_emit_read = nullptr,
                           const std::function<void()>& drain = {}) {
  clear_error();
  if (!g || !out) return set_error(MBE_ERR_INVALID, "null argument");
  memset(out, 0, sizeof(*out));
  mbe_params prm;
  if (params) prm = *params;
  else mbe_params_default(&prm);
  const double t0 = now_s();  // reference exe_time_ starts at Execute() (src/IterFinderGpu.cu:1096)
  CK(cudaSetDevice(g->device));
  const HostGraph& h = g->h;
  int32_t rb = prm.root_begin, re = prm.root_end;
  if (rb == 0 && re == 0) re = h.V_size;
  if (rb < 0 || re > h.V_size || rb > re)
    return set_error(MBE_ERR_INVALID, "root range [%d,%d) outside [0,%d)", rb, re, h.V_size);
  int32_t sc = prm.shard_count > 1 ? prm.shard_count : 1;
  int32_t si = prm.shard_count > 1 ? prm.shard_index : 0;
  if (si < 0 || si >= sc) return set_error(MBE_ERR_INVALID, "shard_index %d outside [0,%d)", si, sc);
  int32_t span = re - rb;
  int32_t n_roots = span > si ? (span - si + sc - 1) / sc : 0;

  DevGraph dg;
  memset(&dg, 0, sizeof(dg));
  dg.nV = h.V_size;
  dg.nU = h.U_size;
  dg.nE = h.edge_size;
  dg.row_off = g->d_row_off;
  dg.col = g->d_col;
  dg.rev_off = g->d_rev_off;
  dg.rev_col = g->d_rev_col;
  dg.ukey = g->d_ukey;
  dg.vkey = g->d_vkey;
  dg.swapped = h.swapped;
  dg.root_end = re;
  dg.root_offset = si;
  dg.root_stride = sc;
  dg.n_roots = n_roots;
  int rc = apply_tuning(prm, &dg);
  if (rc) return rc;

  Workspace& ws = g_ws[g->device];
  std::lock_guard<std::mutex> lock(ws.mu);
  LaunchSpec spec;
  spec.device = g->device;
  spec.map_words = std::max<int32_t>(h.V_size, 1);
  spec.capC = std::max<int32_t>(1, std::min<int32_t>(h.V_size, g->capS));
  spec.capL = g->capL;
  spec.capS = g->capS;
  spec.n_graphs = 1;
  std::vector<int32_t> big_list;
  std::vector<uint8_t> big_flags;
  if ((rc = plan_two_tiers(g, prm, rb, re, si, sc, n_roots, ws.scratch_bytes, &spec, &big_list,
                           &big_flags)))
    return rc;
  LaunchPlan plan;
  if ((rc = engine_prepare(ws, spec, prm, &plan))) return rc;
  plan.ep.emit = d_emit;
  plan.ep.emit_cap = emit_cap;
  plan.ep.emit_read = d_emit_read;
  if (plan.ep.n_big_warps > 0) {
    if (big_list.size() > ws.big_roots_cap) {
      cudaFree(ws.big_roots);
      ws.big_roots = nullptr;
      ws.big_roots_cap = 0;
      CK(cudaMalloc((void**)&ws.big_roots, sizeof(int32_t) * big_list.size()));
      ws.big_roots_cap = big_list.size();
    }
    if (big_flags.size() > ws.big_flag_cap) {
      cudaFree(ws.big_flag);
      ws.big_flag = nullptr;
      ws.big_flag_cap = 0;
      CK(cudaMalloc((void**)&ws.big_flag, big_flags.size()));
      ws.big_flag_cap = big_flags.size();
    }
    if (big_list.size() > ws.big_parts_cap) {
      cudaFree(ws.big_parts);
      ws.big_parts = nullptr;
      ws.big_parts_cap = 0;
      CK(cudaMalloc((void**)&ws.big_parts, 4 * sizeof(int32_t) * big_list.size()));
      ws.big_parts_cap = big_list.size();
    }
    CK(cudaMemcpyAsync(ws.big_roots, big_list.data(), sizeof(int32_t) * big_list.size(),
                       cudaMemcpyHostToDevice, 0));
    CK(cudaMemcpyAsync(ws.big_flag, big_flags.data(), big_flags.size(), cudaMemcpyHostToDevice, 0));
    CK(cudaMemsetAsync(ws.big_parts, 0, 4 * sizeof(int32_t) * big_list.size(), 0));
    plan.ep.n_big_roots = (int32_t)big_list.size();
    plan.ep.big_roots = ws.big_roots;
    plan.ep.big_flag = ws.big_flag;
    plan.ep.big_parts = ws.big_parts;
    plan.ep.big_parts_cap = (int32_t)big_list.size();
  }
  if (prm.l2_window >= 0) {
    // The persisting L2 limit is a setting of this process's context (the
    // device's own configuration is untouched); set once per device.
    if (ws.l2_persist < 0) {
      int persist = 0, maxw = 0;
      CK(cudaDeviceGetAttribute(&persist, cudaDevAttrMaxPersistingL2CacheSize, g->device));
      CK(cudaDeviceGetAttribute(&maxw, cudaDevAttrMaxAccessPolicyWindowSize, g->device));
      ws.l2_persist = persist > 0 && maxw > 0 ? persist : 0;
      ws.l2_max_window = maxw;
      if (ws.l2_persist > 0) CK(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, (size_t)persist));
    }
    const size_t bytes = std::min<size_t>(sizeof(int32_t) * (size_t)h.edge_size,
                                          (size_t)ws.l2_max_window);
    if (ws.l2_persist > 0 && bytes > 0) {
      plan.l2_base = g->d_rev_col;
      plan.l2_bytes = bytes;
      plan.l2_hit = (float)std::min(1.0, (double)ws.l2_persist / (double)bytes);
    }
  }
  long long prefix[2] = {0, n_roots};
  CK(cudaMemcpyAsync(ws.d_graph1, &dg, sizeof(dg), cudaMemcpyHostToDevice, 0));
  CK(cudaMemcpyAsync(ws.d_prefix1, prefix, sizeof(prefix), cudaMemcpyHostToDevice, 0));
  if ((rc = engine_enqueue(ws, &plan, ws.d_graph1, ws.d_prefix1, ws.d_gres1, 1, 0, ws.ev0, ws.ev1)))
    return rc;
  if (drain) {
    // Producers may wait for room in the ring: drain it while the launch runs.
    while (true) {
      drain();
      const cudaError_t q = cudaEventQuery(ws.ev1);
      if (q == cudaSuccess) break;
      if (q != cudaErrorNotReady) return cuda_fail(q, "waiting for the launch");
      std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
  }
  EnumCtl ctl;
  unsigned long long gres[3];
  CK(cudaMemcpy(&ctl, ws.ctl, sizeof(EnumCtl), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(gres, ws.d_gres1, sizeof(gres), cudaMemcpyDeviceToHost));
  if (plan.l2_bytes > 0) CK(cudaCtxResetPersistingL2Cache());  // later work gets the L2 back
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, ws.ev0, ws.ev1));
  out->count = gres[0];
  out->set_hash = gres[1];
  out->non_maximal = gres[2];
  out->kernel_ms = ms;
  fill_profile(ctl, out);
  if (prm.sm_timing) {
    const int blocks = plan.blocks;
    std::vector<unsigned long long> ex(2 * (size_t)blocks);
    CK(cudaMemcpy(ex.data(), ws.exit_ns, 2 * sizeof(unsigned long long) * blocks,
                  cudaMemcpyDeviceToHost));
    auto mm = std::minmax_element(ex.begin(), ex.begin() + blocks);
    out->sm_exit_min_ms = *mm.first / 1e6;
    out->sm_exit_max_ms = *mm.second / 1e6;
    double busy = 0;
    for (int b = 0; b < blocks; ++b) busy += (double)ex[blocks + b];
    out->warp_busy_frac = ms > 0 ? busy / 1e6 / ((double)plan.warps * ms) : 0.0;
  }
  out->enum_seconds = now_s() - t0;
  if (emit_pos) *emit_pos = ctl.emit_pos;
  return engine_status(ws, ctl);
}

int mbe_enumerate(mbe_graph* g, const mbe_params* params, mbe_result* out) {
  return enumerate_graph(g, params, out, nullptr, 0, nullptr);
}

}  // extern "C"

// One record of the device ring -> the biclique in original ids and sides:
// L (internal U ids) as given, R = N(L) from the internal U -> V lists.
void gmbe::decode_biclique(const HostGraph& h, std::vector<int32_t>& L, std::vector<int32_t>* us,
                           std::vector<int32_t>* vs, std::vector<int32_t>& R,
                           std::vector<int32_t>& tmp) {
  int32_t best = L[0];
  for (int32_t u : L)
    if (h.rev_off[u + 1] - h.rev_off[u] < h.rev_off[best + 1] - h.rev_off[best]) best = u;
  R.assign(h.rev_col.begin() + h.rev_off[best], h.rev_col.begin() + h.rev_off[best + 1]);
  for (int32_t u : L) {
    if (u == best) continue;
    tmp.clear();
    std::set_intersection(R.begin(), R.end(), h.rev_col.begin() + h.rev_off[u],
                          h.rev_col.begin() + h.rev_off[u + 1], std::back_inserter(tmp));
    R.swap(tmp);
  }
  us->clear();
  vs->clear();
  for (int32_t u : L) (h.swapped ? vs : us)->push_back(h.u_orig[u]);
  for (int32_t v : R) (h.swapped ? us : vs)->push_back(h.v_orig[v]);
  std::sort(us->begin(), us->end());
  std::sort(vs->begin(), vs->end());
}

extern "C" {

extern "C" int mbe_enumerate_emit_stream(mbe_graph* g, const mbe_params* params, mbe_result* out,
                                         int64_t ring_words, mbe_emit_fn fn, void* user) {
  clear_error();
  if (!g || !out || !fn) return set_error(MBE_ERR_INVALID, "null argument");
  CK(cudaSetDevice(g->device));
  int rc;
  if ((rc = ensure_host_csr(g))) return rc;
  // The ring holds at least one record of the largest L (a root's degree).
  const long long cap = std::max<long long>({ring_words, (long long)g->capL + 2, 64});
  int32_t* h_ring = nullptr;
  unsigned long long* h_read = nullptr;
  int32_t* d_ring = nullptr;
  unsigned long long* d_read = nullptr;
  cudaError_t e = cudaHostAlloc((void**)&h_ring, sizeof(int32_t) * (size_t)cap, cudaHostAllocMapped);
  if (e == cudaSuccess) e = cudaHostAlloc((void**)&h_read, sizeof(unsigned long long), cudaHostAllocMapped);
  if (e == cudaSuccess) {
    memset(h_ring, 0, sizeof(int32_t) * (size_t)cap);
    *h_read = 0;
    e = cudaHostGetDevicePointer((void**)&d_ring, h_ring, 0);
  }
  if (e == cudaSuccess) e = cudaHostGetDevicePointer((void**)&d_read, h_read, 0);
  if (e != cudaSuccess) {
    if (h_ring) cudaFreeHost(h_ring);
    if (h_read) cudaFreeHost(h_read);
    return set_error(MBE_ERR_NOMEM, "emission ring of %lld words: %s", cap, cudaGetErrorString(e));
  }
  const HostGraph& h = g->h;
  unsigned long long consumed = 0;
  bool stopped = false;
  std::vector<int32_t> L, R, tmp, us, vs;
  auto drain = [&]() {
    volatile int32_t* r = h_ring;
    while (true) {
      const int32_t len = r[consumed % (unsigned long long)cap];
      if (len <= 0) return;
      L.resize((size_t)len);
      for (int32_t i = 0; i < len; ++i) L[i] = r[(consumed + 2 + i) % (unsigned long long)cap];
      for (int32_t i = 0; i < len + 2; ++i) r[(consumed + i) % (unsigned long long)cap] = 0;
      consumed += (unsigned long long)len + 2;
      *(volatile unsigned long long*)h_read = consumed;
      if (!stopped) {
        decode_biclique(h, L, &us, &vs, R, tmp);
        if (fn(us.data(), (int32_t)us.size(), vs.data(), (int32_t)vs.size(), user) != 0)
          stopped = true;
      }
    }
  };
  unsigned long long reserved = 0;
  rc = enumerate_graph(g, params, out, d_ring, cap, &reserved, d_read, drain);
  if (rc == MBE_OK) {
    // Every reserved record is committed once the launch has ended.
    while (consumed < reserved) drain();
  }
  cudaFreeHost(h_ring);
  cudaFreeHost(h_read);
  return rc;
}

extern "C" int mbe_enumerate_emit(mbe_graph* g, const mbe_params* params, mbe_result* out,
                                  int32_t* buf, int64_t buf_words, int64_t* used_words) {
  clear_error();
  if (!g || !out || !used_words || buf_words < 0 || (buf_words > 0 && !buf))
    return set_error(MBE_ERR_INVALID, "null or negative argument");
  *used_words = 0;
  struct Sink {
    int32_t* buf;
    int64_t cap, used;
    bool full;
  } sink{buf, buf_words, 0, false};
  auto put = [](const int32_t* u, int32_t nu, const int32_t* v, int32_t nv, void* p) -> int {
    Sink* s = static_cast<Sink*>(p);
    const int64_t need = 2 + (int64_t)nu + nv;
    if (s->used + need > s->cap) {
      s->full = true;
      return 1;  // stop delivering; the enumeration still completes
    }
    s->buf[s->used] = nu;
    s->buf[s->used + 1] = nv;
    std::copy(u, u + nu, s->buf + s->used + 2);
    std::copy(v, v + nv, s->buf + s->used + 2 + nu);
    s->used += need;
    return 0;
  };
  int rc = mbe_enumerate_emit_stream(g, params, out, int64_t(1) << 22, put, &sink);
  *used_words = sink.used;
  if (rc) return rc;
  if (sink.full)
    return set_error(MBE_ERR_CAPACITY, "record buffer of %lld words too small", (long long)buf_words);
  return MBE_OK;
}

}  // extern "C"
