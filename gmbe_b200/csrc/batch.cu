// Batched enumeration: many graphs in one persistent launch.
//
// All graphs of a batch live in one device arena (one allocation per array
// kind) with a descriptor per graph.  A run is one launch of the enumeration
// kernel over every graph: warps claim (graph, root) positions from a single
// counter over the graphs' root lists laid end to end (graphs ordered by
// estimated work, heaviest first), results land in per-graph slots, and
// heavy subtrees are shared through the same sub-problem export as a single
// graph.  The launch sequence (clears, kernel, result read-back into pinned
// host memory) is captured into a CUDA graph once and replayed; descriptor
// edits (per-graph tuning, which graphs take part) do not need a new capture
// because the kernel reads the descriptors at run time.  No counterpart in
// the reference, which enumerates one graph per process (src/main.cu).
#include <cuda_runtime.h>
#include <sys/time.h>

#include <algorithm>
#include <cstring>
#include <numeric>

#include "engine.h"

using namespace gmbe;

struct mbe_batch {
  int device = 0;
  int32_t n = 0;
  std::vector<int32_t> order;   // descriptor position -> input index
  std::vector<int32_t> pos_of;  // input index -> descriptor position
  std::vector<DevGraph> hg;     // descriptors (position order)
  std::vector<int32_t> all_roots;
  std::vector<double> cost;     // estimated work: sum over roots of the two-hop multiset
  int32_t* d_i32 = nullptr;
  uint64_t* d_keys = nullptr;
  DevGraph* d_graphs = nullptr;
  long long* d_prefix = nullptr;
  unsigned long long* d_gres = nullptr;
  unsigned long long* h_gres = nullptr;  // pinned
  EnumCtl* h_ctl = nullptr;              // pinned
  LaunchSpec spec;
  bool desc_dirty = true;
  cudaStream_t stream = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t exec_gen = 0;
  mbe_params exec_prm;
  int exec_warps = 0;
};

namespace {

#define BCK(call)                                                                         \
  do {                                                                                    \
    cudaError_t _e = (call);                                                              \
    if (_e != cudaSuccess) return set_error(MBE_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(_e)); \
  } while (0)

double now_ms() {
  struct timeval tv;
  gettimeofday(&tv, nullptr);
  return (double)tv.tv_sec * 1e3 + (double)tv.tv_usec * 1e-3;
}

void batch_release(mbe_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->stream) cudaStreamDestroy(b->stream);
  cudaFree(b->d_i32);
  cudaFree(b->d_keys);
  cudaFree(b->d_graphs);
  cudaFree(b->d_prefix);
  cudaFree(b->d_gres);
  cudaFreeHost(b->h_gres);
  cudaFreeHost(b->h_ctl);
  b->exec = nullptr;
  b->stream = nullptr;
  b->d_i32 = nullptr;
  b->d_keys = nullptr;
  b->d_graphs = nullptr;
  b->d_prefix = nullptr;
  b->d_gres = nullptr;
  b->h_gres = nullptr;
  b->h_ctl = nullptr;
}

// Uploads descriptors and the root prefix (roots of positions whose active
// flag is clear count as zero).
int upload_descriptors(mbe_batch* b, const std::vector<char>* active) {
  std::vector<DevGraph> d = b->hg;
  std::vector<long long> prefix(b->n + 1, 0);
  for (int32_t i = 0; i < b->n; ++i) {
    if (active && !(*active)[i]) d[i].n_roots = 0;
    prefix[i + 1] = prefix[i] + d[i].n_roots;
  }
  BCK(cudaMemcpyAsync(b->d_graphs, d.data(), sizeof(DevGraph) * b->n, cudaMemcpyHostToDevice,
                      b->stream));
  BCK(cudaMemcpyAsync(b->d_prefix, prefix.data(), sizeof(long long) * (b->n + 1),
                      cudaMemcpyHostToDevice, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  b->desc_dirty = active != nullptr;
  return MBE_OK;
}

bool same_global(const mbe_params& a, const mbe_params& c) {
  return a.prune == c.prune && a.blocks == c.blocks && a.queue_capacity == c.queue_capacity &&
         a.wait_limit_ns == c.wait_limit_ns && a.split_mode == c.split_mode &&
         a.root_split_size == c.root_split_size && a.share_min_work == c.share_min_work &&
         a.range_split_work == c.range_split_work && a.range_chunk == c.range_chunk &&
         a.eager_share == c.eager_share && a.time_limit_ns == c.time_limit_ns &&
         a.touch_scan == c.touch_scan && a.slot_records == c.slot_records &&
         a.share_counts == c.share_counts && a.l2_window == c.l2_window;
}

// Captures (or re-captures) the launch when the workspace or the global
// parameters changed since the last capture.  Caller holds the workspace lock.
int ensure_captured(mbe_batch* b, Workspace& ws, const mbe_params& prm) {
  if (b->exec && b->exec_gen == ws.gen && same_global(prm, b->exec_prm)) return MBE_OK;
  LaunchPlan plan;
  int rc = engine_prepare(ws, b->spec, prm, &plan);
  if (rc) return rc;
  if ((rc = engine_clear_maps(ws, &plan, b->stream))) return rc;
  BCK(cudaStreamSynchronize(b->stream));
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  cudaGraph_t graph = nullptr;
  BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  rc = engine_enqueue(ws, &plan, b->d_graphs, b->d_prefix, b->d_gres, b->n, b->stream, nullptr,
                      nullptr);
  cudaError_t e1 = cudaMemcpyAsync(b->h_gres, b->d_gres, 3 * sizeof(unsigned long long) * b->n,
                                   cudaMemcpyDeviceToHost, b->stream);
  cudaError_t e2 = cudaMemcpyAsync(b->h_ctl, ws.ctl, sizeof(EnumCtl), cudaMemcpyDeviceToHost,
                                   b->stream);
  cudaError_t e3 = cudaStreamEndCapture(b->stream, &graph);
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return set_error(MBE_ERR_CUDA, "capturing the batch launch failed");
  }
  cudaError_t e4 = cudaGraphInstantiate(&b->exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e4 != cudaSuccess) {
    b->exec = nullptr;
    return set_error(MBE_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e4));
  }
  b->exec_gen = ws.gen;
  b->exec_prm = prm;
  b->exec_warps = plan.warps;
  return MBE_OK;
}

// One replay; fills per-position results into h_gres and the control block.
int replay(mbe_batch* b, Workspace& ws, float* kernel_ms) {
  BCK(cudaEventRecord(ws.ev0, b->stream));
  BCK(cudaGraphLaunch(b->exec, b->stream));
  BCK(cudaEventRecord(ws.ev1, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  BCK(cudaEventElapsedTime(kernel_ms, ws.ev0, ws.ev1));
  return engine_status(ws, *b->h_ctl);
}

}  // namespace

extern "C" {

int mbe_batch_from_csr(int32_t n, const int32_t* const* row_offs, const int32_t* const* cols,
                       const int32_t* nVs, const int32_t* nUs, const int64_t* nEs,
                       const mbe_opts* opts, mbe_batch** out) {
  clear_error();
  if (!out || n <= 0 || !row_offs || !cols || !nVs || !nEs)
    return set_error(MBE_ERR_INVALID, "null or empty batch");
  *out = nullptr;
  mbe_opts o;
  if (opts) o = *opts;
  else mbe_opts_default(&o);
  std::vector<HostGraph> hosts(n);
  std::vector<int32_t> capL(n), capS(n);
  mbe_batch* b = new mbe_batch();
  b->device = o.device;
  b->n = n;
  b->cost.assign(n, 0.0);
  for (int32_t i = 0; i < n; ++i) {
    int rc = build_host_graph(row_offs[i], cols[i], nVs[i], nUs ? nUs[i] : 0, nEs[i], o, &hosts[i]);
    if (!rc) rc = graph_caps(hosts[i], &capL[i], &capS[i]);
    if (rc) {
      delete b;
      return set_error(rc, "graph %d: %s", i, mbe_last_error_string());
    }
    const HostGraph& h = hosts[i];
    double c = 0;
    for (int32_t u = 0; u < h.U_size; ++u) {
      double d = h.rev_off[u + 1] - h.rev_off[u];
      c += d * d;
    }
    b->cost[i] = c;
  }
  // Heaviest graphs first, so their roots start at once.
  b->order.resize(n);
  std::iota(b->order.begin(), b->order.end(), 0);
  std::stable_sort(b->order.begin(), b->order.end(),
                   [&](int32_t x, int32_t y) { return b->cost[x] > b->cost[y]; });
  b->pos_of.resize(n);
  for (int32_t p = 0; p < n; ++p) b->pos_of[b->order[p]] = p;
  // Arena: int32 arrays, then uint64 keys.
  size_t n32 = 0, n64 = 0;
  for (const HostGraph& h : hosts) {
    n32 += h.row_off.size() + h.col.size() + h.rev_off.size() + h.rev_col.size();
    n64 += (size_t)h.U_size + h.V_size;
  }
  std::vector<int32_t> a32;
  std::vector<uint64_t> a64;
  a32.reserve(n32);
  a64.reserve(n64);
  struct Off {
    size_t ro, co, rro, rco, uk, vk;
  };
  std::vector<Off> offs(n);
  for (int32_t p = 0; p < n; ++p) {
    const HostGraph& h = hosts[b->order[p]];
    Off& f = offs[p];
    f.ro = a32.size();
    a32.insert(a32.end(), h.row_off.begin(), h.row_off.end());
    f.co = a32.size();
    a32.insert(a32.end(), h.col.begin(), h.col.end());
    f.rro = a32.size();
    a32.insert(a32.end(), h.rev_off.begin(), h.rev_off.end());
    f.rco = a32.size();
    a32.insert(a32.end(), h.rev_col.begin(), h.rev_col.end());
    std::vector<uint64_t> uk, vk;
    host_keys(h, &uk, &vk);
    f.uk = a64.size();
    a64.insert(a64.end(), uk.begin(), uk.end());
    f.vk = a64.size();
    a64.insert(a64.end(), vk.begin(), vk.end());
  }
  cudaError_t e;
  if ((e = cudaSetDevice(b->device)) != cudaSuccess ||
      (e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaMalloc((void**)&b->d_i32, sizeof(int32_t) * std::max<size_t>(a32.size(), 1))) !=
          cudaSuccess ||
      (e = cudaMalloc((void**)&b->d_keys, sizeof(uint64_t) * std::max<size_t>(a64.size(), 1))) !=
          cudaSuccess ||
      (e = cudaMalloc((void**)&b->d_graphs, sizeof(DevGraph) * n)) != cudaSuccess ||
      (e = cudaMalloc((void**)&b->d_prefix, sizeof(long long) * (n + 1))) != cudaSuccess ||
      (e = cudaMalloc((void**)&b->d_gres, 3 * sizeof(unsigned long long) * n)) != cudaSuccess ||
      (e = cudaMallocHost((void**)&b->h_gres, 3 * sizeof(unsigned long long) * n)) != cudaSuccess ||
      (e = cudaMallocHost((void**)&b->h_ctl, sizeof(EnumCtl))) != cudaSuccess ||
      (e = cudaMemcpy(b->d_i32, a32.data(), sizeof(int32_t) * a32.size(), cudaMemcpyHostToDevice)) !=
          cudaSuccess ||
      (e = cudaMemcpy(b->d_keys, a64.data(), sizeof(uint64_t) * a64.size(),
                      cudaMemcpyHostToDevice)) != cudaSuccess) {
    batch_release(b);
    delete b;
    return set_error(MBE_ERR_NOMEM, "batch arena: %s", cudaGetErrorString(e));
  }
  mbe_params def;
  mbe_params_default(&def);
  b->hg.resize(n);
  b->all_roots.resize(n);
  LaunchSpec& sp = b->spec;
  sp.device = b->device;
  sp.n_graphs = n;
  sp.map_words = 1;
  sp.capC = sp.capL = sp.capS = 1;
  for (int32_t p = 0; p < n; ++p) {
    const int32_t i = b->order[p];
    const HostGraph& h = hosts[i];
    DevGraph& dg = b->hg[p];
    memset(&dg, 0, sizeof(dg));
    dg.nV = h.V_size;
    dg.nU = h.U_size;
    dg.nE = h.edge_size;
    dg.row_off = b->d_i32 + offs[p].ro;
    dg.col = b->d_i32 + offs[p].co;
    dg.rev_off = b->d_i32 + offs[p].rro;
    dg.rev_col = b->d_i32 + offs[p].rco;
    dg.ukey = b->d_keys + offs[p].uk;
    dg.vkey = b->d_keys + offs[p].vk;
    dg.swapped = h.swapped;
    dg.root_end = h.V_size;
    dg.root_offset = 0;
    dg.root_stride = 1;
    dg.n_roots = h.V_size;
    b->all_roots[p] = h.V_size;
    apply_tuning(def, &dg);
    sp.map_words = std::max(sp.map_words, h.V_size);
    sp.capC = std::max(sp.capC, std::max<int32_t>(1, std::min<int32_t>(h.V_size, capS[i])));
    sp.capL = std::max(sp.capL, capL[i]);
    sp.capS = std::max(sp.capS, capS[i]);
  }
  *out = b;
  return MBE_OK;
}

int mbe_batch_size(const mbe_batch* b) { return b ? b->n : 0; }

int mbe_batch_set_tuning(mbe_batch* b, int32_t index, const mbe_params* p) {
  clear_error();
  if (!b || !p || index < -1 || index >= b->n) return set_error(MBE_ERR_INVALID, "bad argument");
  for (int32_t i = (index < 0 ? 0 : index); i < (index < 0 ? b->n : index + 1); ++i) {
    int rc = apply_tuning(*p, &b->hg[b->pos_of[i]]);
    if (rc) return rc;
  }
  b->desc_dirty = true;
  return MBE_OK;
}

int mbe_batch_get_tuning(const mbe_batch* b, int32_t index, mbe_params* out) {
  clear_error();
  if (!b || !out || index < 0 || index >= b->n) return set_error(MBE_ERR_INVALID, "bad argument");
  const DevGraph& dg = b->hg[b->pos_of[index]];
  mbe_params_default(out);
  out->bound_height = dg.bound_height;
  out->bound_size = dg.bound_size;
  out->bitmap_max_l = dg.tier2_max_l;
  out->direct_max_c = dg.direct_max_c;
  return MBE_OK;
}

int mbe_batch_run(mbe_batch* b, const mbe_params* params, mbe_result* per_graph, mbe_result* total) {
  clear_error();
  if (!b) return set_error(MBE_ERR_INVALID, "null batch");
  const double t0 = now_ms();
  mbe_params prm;
  if (params) prm = *params;
  else mbe_params_default(&prm);
  BCK(cudaSetDevice(b->device));
  Workspace& ws = workspace(b->device);
  std::lock_guard<std::mutex> lock(ws.mu);
  int rc;
  if (b->desc_dirty && (rc = upload_descriptors(b, nullptr))) return rc;
  if ((rc = ensure_captured(b, ws, prm))) return rc;
  float ms = 0;
  rc = replay(b, ws, &ms);
  if (per_graph) {
    for (int32_t i = 0; i < b->n; ++i) {
      const int32_t p = b->pos_of[i];
      memset(&per_graph[i], 0, sizeof(mbe_result));
      per_graph[i].count = b->h_gres[3 * p];
      per_graph[i].set_hash = b->h_gres[3 * p + 1];
      per_graph[i].non_maximal = b->h_gres[3 * p + 2];
      per_graph[i].status = b->h_ctl->status;
    }
  }
  if (total) {
    memset(total, 0, sizeof(*total));
    for (int32_t p = 0; p < b->n; ++p) {
      total->count += b->h_gres[3 * p];
      total->set_hash += b->h_gres[3 * p + 1];
      total->non_maximal += b->h_gres[3 * p + 2];
    }
    total->kernel_ms = ms;
    fill_profile(*b->h_ctl, total);
    if (total->max_task_graph >= 0 && total->max_task_graph < b->n)
      total->max_task_graph = b->order[total->max_task_graph];  // input index
    total->enum_seconds = (now_ms() - t0) / 1e3;
  }
  return rc;
}

int mbe_batch_autotune(mbe_batch* b, const mbe_params* params, int32_t n_classes,
                       int32_t* chosen) {
  clear_error();
  if (!b || n_classes < 1 || n_classes > 64) return set_error(MBE_ERR_INVALID, "bad argument");
  mbe_params prm;
  if (params) prm = *params;
  else mbe_params_default(&prm);
  // Candidate tunings (results never depend on them): split bounds, the
  // bitmap-tier limit on |L| and the direct-entry limit on |C|.
  const int32_t cand[][4] = {
      {20, 1500, 128, 4096}, {5, 200, 128, 4096},   {20, 15000, 128, 1024},
      {50, 1500, 64, 16384}, {1 << 30, 1 << 30, 128, 4096}, {10, 500, 128, 16384},
  };
  const int n_cand = (int)(sizeof(cand) / sizeof(cand[0]));
  // Size classes: quantiles of estimated work over the batch (positions are
  // already sorted by work, heaviest first).
  std::vector<int32_t> cls(b->n);
  for (int32_t p = 0; p < b->n; ++p) cls[p] = (int32_t)((int64_t)p * n_classes / b->n);
  BCK(cudaSetDevice(b->device));
  Workspace& ws = workspace(b->device);
  std::lock_guard<std::mutex> lock(ws.mu);
  int rc;
  if ((rc = upload_descriptors(b, nullptr))) return rc;
  if ((rc = ensure_captured(b, ws, prm))) return rc;
  std::vector<unsigned long long> ref(3 * (size_t)b->n);
  for (int32_t c = 0; c < n_classes; ++c) {
    std::vector<char> active(b->n, 0);
    int members = 0;
    for (int32_t p = 0; p < b->n; ++p)
      if (cls[p] == c) {
        active[p] = 1;
        ++members;
      }
    if (!members) continue;
    double best_ms = 1e300;
    int best = 0;
    for (int k = 0; k < n_cand; ++k) {
      mbe_params t = prm;
      t.bound_height = cand[k][0];
      t.bound_size = cand[k][1];
      t.bitmap_max_l = cand[k][2];
      t.direct_max_c = cand[k][3];
      for (int32_t p = 0; p < b->n; ++p)
        if (active[p]) apply_tuning(t, &b->hg[p]);
      if ((rc = upload_descriptors(b, &active))) return rc;
      float ms = 0, best_k = 1e30f;
      for (int rep = 0; rep < 2; ++rep) {
        if ((rc = replay(b, ws, &ms))) return rc;
        best_k = std::min(best_k, ms);
      }
      // Every candidate must give the same per-graph results.
      // (count and set hash; the non-maximal count depends on the tuning)
      for (int32_t p = 0; p < b->n; ++p) {
        if (!active[p]) continue;
        for (int f = 0; f < 2; ++f) {
          if (k == 0) ref[3 * p + f] = b->h_gres[3 * p + f];
          else if (ref[3 * p + f] != b->h_gres[3 * p + f])
            return set_error(MBE_ERR_CUDA, "autotune: results differ between tunings (graph %d)",
                             b->order[p]);
        }
      }
      if (best_k < best_ms) {
        best_ms = best_k;
        best = k;
      }
    }
    mbe_params t = prm;
    t.bound_height = cand[best][0];
    t.bound_size = cand[best][1];
    t.bitmap_max_l = cand[best][2];
    t.direct_max_c = cand[best][3];
    for (int32_t p = 0; p < b->n; ++p)
      if (cls[p] == c) apply_tuning(t, &b->hg[p]);
    if (chosen) chosen[c] = best;
  }
  return upload_descriptors(b, nullptr);
}

int mbe_batch_free(mbe_batch* b) {
  clear_error();
  if (!b) return MBE_OK;
  cudaSetDevice(b->device);
  batch_release(b);
  delete b;
  return MBE_OK;
}

}  // extern "C"
