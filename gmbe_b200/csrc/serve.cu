// Serving: continuous batching of enumeration requests on one GPU.
//
// A request's graph is prepared on the host by the submitting thread (-t/-o,
// both CSRs, hash keys, capacities), laid out as one arena block image, and
// queued.  The server thread admits queued graphs first come, first served
// while arena space and graph slots last: it copies the block into the arena
// (copy stream), appends its block index to the arrival ring and raises the
// published count.  The persistent kernel (server mode of mbe_enum_kernel)
// claims roots from the oldest published graph with roots left, shares work
// between all resident graphs, and writes a completion record into host-mapped
// memory when a graph's last task finishes.  The server thread collects those
// records, and launches again whenever graphs are resident and no launch runs
// (a launch ends once idle for idle_exit_ns).  Arena blocks are bump-allocated
// and the arena rewinds only when nothing is resident and no launch runs, so no
// address is rewritten while a launch may hold it in a cache.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.h"
#include "enum_launch.h"
#include "internal.h"
#include "mbe.h"

using namespace gmbe;

namespace {

constexpr size_t kBlock = size_t(1) << kServeBlockShift;
constexpr size_t kArrayAlign = 256;

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

enum ReqState { kWaiting, kResident, kDone, kFailed, kCancelled };

struct Request {
  uint64_t id = 0;
  ReqState state = kWaiting;
  std::vector<char> image;  // the arena block; descriptor pointers patched on admission
  size_t bytes = 0;         // image size, a multiple of kBlock
  size_t o_row_off = 0, o_col = 0, o_rev_off = 0, o_rev_col = 0, o_ukey = 0, o_vkey = 0;
  size_t arena_off = 0;  // where it was placed, once admitted
  DevGraph dg;
  double t_submit = 0;
  mbe_result res;
  int rc = MBE_OK;
};

}  // namespace

struct mbe_server {
  int device = 0;
  mbe_server_config cfg;
  mbe_params prm;
  // Device side.
  char* d_arena = nullptr;
  size_t bump = 0;
  ServeCtl* d_sctl = nullptr;
  uint32_t* d_arr_blk = nullptr;
  int32_t arr_cap = 0;
  ServeDone* h_done = nullptr;  // host-mapped completion ring
  ServeDone* d_done = nullptr;
  int32_t done_cap = 0;
  EnumCtl* d_ctl = nullptr;
  Task* d_q_tasks = nullptr;
  unsigned long long* d_q_seq = nullptr;
  int32_t q_cap = 0;
  int32_t* d_slots = nullptr;
  uint32_t* d_slot_bits = nullptr;
  int32_t nslot = 0;
  int32_t* d_scratch = nullptr;
  int blocks = 0;
  ScratchLayout sl;
  EnumParams ep;
  int32_t capC = 1, capL = 1, capS = 1, map_words = 1;
  cudaStream_t s_run = nullptr, s_copy = nullptr, s_peek = nullptr;
  cudaEvent_t ev_run = nullptr, ev_copy = nullptr;
  bool running = false;
  // Host side, under mu.
  std::mutex mu;
  std::condition_variable cv_loop, cv_done;
  std::deque<Request*> waiting;
  std::unordered_map<uint64_t, Request*> reqs;
  uint64_t next_id = 1;
  uint64_t published = 0, collected = 0;
  int64_t resident = 0;
  bool stopping = false;
  int fatal = MBE_OK;
  std::string fatal_msg;
  mbe_server_stats st;
  std::thread loop;
};

namespace {

#define SCK(call)                                                                          \
  do {                                                                                     \
    cudaError_t _e = (call);                                                               \
    if (_e != cudaSuccess)                                                                 \
      return set_error(MBE_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(_e));             \
  } while (0)

void release(mbe_server* s) {
  cudaSetDevice(s->device);
  if (s->s_run) cudaStreamSynchronize(s->s_run);
  if (s->s_copy) cudaStreamSynchronize(s->s_copy);
  cudaFree(s->d_arena);
  cudaFree(s->d_sctl);
  cudaFree(s->d_arr_blk);
  if (s->h_done) cudaFreeHost(s->h_done);
  cudaFree(s->d_ctl);
  cudaFree(s->d_q_tasks);
  cudaFree(s->d_q_seq);
  cudaFree(s->d_slots);
  cudaFree(s->d_slot_bits);
  cudaFree(s->d_scratch);
  if (s->ev_run) cudaEventDestroy(s->ev_run);
  if (s->ev_copy) cudaEventDestroy(s->ev_copy);
  if (s->s_run) cudaStreamDestroy(s->s_run);
  if (s->s_copy) cudaStreamDestroy(s->s_copy);
  if (s->s_peek) cudaStreamDestroy(s->s_peek);
  for (auto& kv : s->reqs) delete kv.second;
  s->reqs.clear();
}

int allocate(mbe_server* s) {
  SCK(cudaSetDevice(s->device));
  const mbe_server_config& c = s->cfg;
  s->map_words = std::max(c.max_v, 1);
  s->capL = std::max(c.max_degree, 1);
  s->capS = std::max(c.max_two_hop, 1);
  s->capC = std::max<int32_t>(1, std::min(s->map_words, s->capS));
  int dev_sms = 0, occ = 0;
  SCK(cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, s->device));
  SCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, mbe_enum_kernel, kEnumThreads, 0));
  if (occ < 1) return set_error(MBE_ERR_CUDA, "enumeration kernel cannot be resident");
  s->blocks = s->prm.blocks > 0 ? std::min(s->prm.blocks, dev_sms * occ) : dev_sms * occ;
  const int warps = s->blocks * kEnumWarps;
  s->sl = make_layout(s->map_words, s->capC, s->capL, s->capS);
  SCK(cudaFuncSetAttribute(mbe_enum_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)enum_smem_bytes(s->sl)));
  const size_t scratch = (size_t)s->sl.words_per_warp * warps * sizeof(int32_t);
  SCK(cudaMalloc((void**)&s->d_scratch, scratch));
  // Every warp's count map starts all-zero; each task leaves it so.
  SCK(cudaMemset2D(s->d_scratch, (size_t)s->sl.words_per_warp * sizeof(int32_t), 0,
                   (size_t)s->sl.zero_words * sizeof(int32_t), (size_t)warps));
  SCK(cudaMalloc((void**)&s->d_arena, (size_t)c.arena_bytes));
  SCK(cudaMalloc((void**)&s->d_sctl, sizeof(ServeCtl)));
  SCK(cudaMemset(s->d_sctl, 0, sizeof(ServeCtl)));
  // Published graphs never outnumber resident ones by more than max_graphs,
  // so a ring of 4 x max_graphs entries is not rewritten while a warp may
  // still read an entry it saw as the head.
  s->arr_cap = 4 * c.max_graphs;
  SCK(cudaMalloc((void**)&s->d_arr_blk, sizeof(uint32_t) * (size_t)s->arr_cap));
  s->done_cap = 2 * c.max_graphs;
  SCK(cudaHostAlloc((void**)&s->h_done, sizeof(ServeDone) * (size_t)s->done_cap,
                    cudaHostAllocMapped));
  memset(s->h_done, 0, sizeof(ServeDone) * (size_t)s->done_cap);
  SCK(cudaHostGetDevicePointer((void**)&s->d_done, s->h_done, 0));
  SCK(cudaMalloc((void**)&s->d_ctl, sizeof(EnumCtl)));
  s->q_cap = s->prm.queue_capacity > 0 ? s->prm.queue_capacity : (1 << 18);
  SCK(cudaMalloc((void**)&s->d_q_tasks, sizeof(Task) * (size_t)s->q_cap));
  SCK(cudaMalloc((void**)&s->d_q_seq, sizeof(unsigned long long) * (size_t)s->q_cap));
  s->nslot = s->prm.split_mode == 1 ? 0 : 4096;
  if (s->nslot) {
    SCK(cudaMalloc((void**)&s->d_slots, sizeof(int32_t) * (size_t)kSlotWordsHost * s->nslot));
    SCK(cudaMalloc((void**)&s->d_slot_bits, sizeof(uint32_t) * (size_t)(s->nslot / 32)));
  }
  SCK(cudaStreamCreateWithFlags(&s->s_run, cudaStreamNonBlocking));
  SCK(cudaStreamCreateWithFlags(&s->s_copy, cudaStreamNonBlocking));
  SCK(cudaStreamCreateWithFlags(&s->s_peek, cudaStreamNonBlocking));
  SCK(cudaEventCreateWithFlags(&s->ev_run, cudaEventDisableTiming));
  SCK(cudaEventCreateWithFlags(&s->ev_copy, cudaEventDisableTiming));
  SCK(cudaDeviceSynchronize());

  EnumParams& ep = s->ep;
  memset(&ep, 0, sizeof(ep));
  ep.prune = s->prm.prune;
  ep.queue_cap = s->q_cap;
  ep.slot_spin_limit = 20000000;
  ep.idle_ns_limit = 600LL * 1000000000LL;
  ep.vertex_split = s->prm.split_mode == 1 ? 1 : 0;
  ep.root_split = s->prm.split_mode == 1 ? 0 : std::max(s->prm.root_split_size, 0);
  ep.share_counts = s->prm.share_counts < 0 ? 0 : 1;
  ep.share_min_work =
      s->prm.share_min_work > 0 ? s->prm.share_min_work : kShareMinWorkDefault;
  apply_range_split(s->prm, &ep.range_work, &ep.range_chunk);
  ep.eager_share = eager_share_of(s->prm);
  ep.server = 1;
  ep.serve.sctl = s->d_sctl;
  ep.serve.arr_blk = s->d_arr_blk;
  ep.serve.done = s->d_done;
  ep.serve.arr_cap = s->arr_cap;
  ep.serve.done_cap = s->done_cap;
  ep.serve.idle_exit_ns = c.idle_exit_ns;
  return MBE_OK;
}

// Starts a launch on the run stream, after the latest arena copies.
int launch(mbe_server* s) {
  SCK(cudaStreamWaitEvent(s->s_run, s->ev_copy, 0));
  SCK(cudaMemsetAsync(s->d_ctl, 0, sizeof(EnumCtl), s->s_run));
  SCK(cudaMemsetAsync(s->d_q_seq, 0, sizeof(unsigned long long) * (size_t)s->q_cap, s->s_run));
  if (s->nslot)
    SCK(cudaMemsetAsync(s->d_slot_bits, 0, sizeof(uint32_t) * (size_t)(s->nslot / 32), s->s_run));
  SlotPool pool;
  memset(&pool, 0, sizeof(pool));  // no large slots in a server
  pool.slots = s->d_slots;
  pool.bits = s->d_slot_bits;
  pool.nslot = s->nslot;
  mbe_enum_kernel<<<s->blocks, kEnumThreads, enum_smem_bytes(s->sl), s->s_run>>>(
      reinterpret_cast<const DevGraph*>(s->d_arena), nullptr, nullptr, s->ep, s->sl, s->d_ctl,
      s->d_q_tasks, s->d_q_seq, pool, s->d_scratch, nullptr);
  SCK(cudaGetLastError());
  SCK(cudaEventRecord(s->ev_run, s->s_run));
  s->running = true;
  s->st.launches++;
  return MBE_OK;
}

void finish(mbe_server* s, Request* r, int rc) {
  r->rc = rc;
  r->state = rc == MBE_OK ? kDone : kFailed;
  r->image.clear();
  r->image.shrink_to_fit();
  s->cv_done.notify_all();
}

// Fails every request not yet finished (a launch failure).
void fail_all(mbe_server* s, int rc) {
  for (auto& kv : s->reqs) {
    Request* r = kv.second;
    if (r->state == kWaiting || r->state == kResident) finish(s, r, rc);
  }
  s->waiting.clear();
  s->resident = 0;
}

// Copies one admitted graph into the arena and publishes it (server thread,
// which holds s->mu on entry and on return).  The arena space, the arrival
// ring position and the request's state are taken under the lock; the copies
// themselves run with the lock released, so that submit, poll and wait are
// never held up behind a graph's staging copy.  The image moves out of the
// request first: nothing another thread does to the request (destroy
// finishing it) touches the memory being copied.
int admit(mbe_server* s, Request* r, std::unique_lock<std::mutex>& lk) {
  const size_t off = s->bump;
  char* base = s->d_arena + off;
  DevGraph& g = r->dg;
  g.row_off = reinterpret_cast<const int32_t*>(base + r->o_row_off);
  g.col = reinterpret_cast<const int32_t*>(base + r->o_col);
  g.rev_off = reinterpret_cast<const int32_t*>(base + r->o_rev_off);
  g.rev_col = reinterpret_cast<const int32_t*>(base + r->o_rev_col);
  g.ukey = reinterpret_cast<const uint64_t*>(base + r->o_ukey);
  g.vkey = reinterpret_cast<const uint64_t*>(base + r->o_vkey);
  ServeGraph hdr;
  memset(&hdr, 0, sizeof(hdr));
  hdr.g = g;
  hdr.pending = (unsigned long long)g.n_roots;
  hdr.request = r->id;
  std::vector<char> image = std::move(r->image);
  r->image = std::vector<char>();
  memcpy(image.data(), &hdr, sizeof(hdr));
  const size_t bytes = r->bytes;
  const uint64_t slot = s->published % (uint64_t)s->arr_cap;
  r->arena_off = off;
  s->bump = off + bytes;
  s->published++;
  s->resident++;
  s->st.admitted++;
  r->state = kResident;
  const uint32_t blk = (uint32_t)(off >> kServeBlockShift);
  const unsigned long long tail = s->published;
  lk.unlock();
  cudaError_t e = cudaMemcpyAsync(base, image.data(), bytes, cudaMemcpyHostToDevice, s->s_copy);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s->d_arr_blk + slot, &blk, sizeof(blk), cudaMemcpyHostToDevice, s->s_copy);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&s->d_sctl->arr_tail, &tail, sizeof(tail), cudaMemcpyHostToDevice,
                        s->s_copy);
  if (e == cudaSuccess) e = cudaEventRecord(s->ev_copy, s->s_copy);
  lk.lock();
  if (e != cudaSuccess)
    return set_error(MBE_ERR_CUDA, "copying a graph to the device: %s", cudaGetErrorString(e));
  return MBE_OK;
}

void server_loop(mbe_server* s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    bool progress = false;
    // Completion records, in the order the device handed out their positions.
    while (true) {
      volatile ServeDone* d = s->h_done + (s->collected % (uint64_t)s->done_cap);
      if (d->seq != s->collected + 1) break;
      const uint64_t id = d->request;
      auto it = s->reqs.find(id);
      if (it != s->reqs.end() && it->second->state == kResident) {
        Request* r = it->second;
        memset(&r->res, 0, sizeof(r->res));
        r->res.count = d->count;
        r->res.set_hash = d->hash;
        r->res.non_maximal = d->non_maximal;
        r->res.enum_seconds = now_s() - r->t_submit;
        s->st.completed++;
        finish(s, r, MBE_OK);
      }
      s->collected++;
      s->resident--;
      progress = true;
    }
    // A launch that ended.
    if (s->running && cudaEventQuery(s->ev_run) == cudaSuccess) {
      s->running = false;
      EnumCtl ctl;
      cudaError_t e = cudaMemcpy(&ctl, s->d_ctl, sizeof(ctl), cudaMemcpyDeviceToHost);
      if (e != cudaSuccess || ctl.status != 0) {
        s->fatal = e != cudaSuccess ? MBE_ERR_CUDA
                                    : (ctl.status == kStCapacity ? MBE_ERR_CAPACITY : MBE_ERR_TIMEOUT);
        s->fatal_msg = e != cudaSuccess ? cudaGetErrorString(e) : "device status";
        fail_all(s, s->fatal);
      }
      progress = true;
    }
    if (!s->running && s->resident == 0 && s->bump != 0) {
      s->bump = 0;  // nothing on the device refers to the arena any more
      s->st.arena_resets++;
    }
    // Admission, first come first served.
    while (!s->waiting.empty() && !s->stopping && s->fatal == MBE_OK) {
      Request* r = s->waiting.front();
      if (s->resident >= s->cfg.max_graphs) break;
      if (s->bump + r->bytes > (size_t)s->cfg.arena_bytes) break;  // rewinds once drained
      s->waiting.pop_front();
      const uint64_t id = r->id;
      int rc = admit(s, r, lk);
      if (rc) {
        s->fatal = rc;
        s->fatal_msg = "copying a graph to the device failed";
        // The lock was released during the copy: look the request up again.
        auto it = s->reqs.find(id);
        if (it != s->reqs.end() && it->second->state == kResident) finish(s, it->second, rc);
        fail_all(s, rc);
        break;
      }
      progress = true;
    }
    if (!s->running && s->resident > 0 && s->fatal == MBE_OK && !s->stopping) {
      int rc = launch(s);
      if (rc) {
        s->fatal = rc;
        s->fatal_msg = "launch failed";
        fail_all(s, rc);
      }
      progress = true;
    }
    if (s->stopping && !s->running) break;
    if (!progress)
      s->cv_loop.wait_for(lk, std::chrono::microseconds(s->running ? 20 : 2000));
  }
}

// Caller holds mu.  Returns the code for a request in its current state and
// forgets it when that state is final.
int take(mbe_server* s, uint64_t id, mbe_result* out) {
  auto it = s->reqs.find(id);
  if (it == s->reqs.end())
    return set_error(MBE_ERR_NOT_FOUND, "unknown request %llu", (unsigned long long)id);
  Request* r = it->second;
  if (r->state == kWaiting || r->state == kResident) return MBE_ERR_AGAIN;
  int rc;
  if (r->state == kDone) {
    if (out) *out = r->res;
    rc = MBE_OK;
  } else if (r->state == kCancelled) {
    rc = set_error(MBE_ERR_CANCELLED, "request %llu was cancelled", (unsigned long long)id);
  } else {
    rc = set_error(r->rc, "request %llu failed: %s", (unsigned long long)id, s->fatal_msg.c_str());
  }
  s->reqs.erase(it);
  delete r;
  return rc;
}

}  // namespace

extern "C" {

void mbe_server_config_default(mbe_server_config* c) {
  if (!c) return;
  memset(c, 0, sizeof(*c));
  c->max_graphs = 4096;
  c->arena_bytes = int64_t(1) << 30;
  c->max_v = 32768;
  c->max_degree = 4096;
  c->max_two_hop = 65536;
  c->idle_exit_ns = 200000;
}

int mbe_server_create(const mbe_server_config* cfg, const mbe_params* params, mbe_server** out) {
  clear_error();
  if (!out) return set_error(MBE_ERR_INVALID, "null output handle");
  *out = nullptr;
  mbe_server_config c;
  mbe_server_config_default(&c);
  if (cfg) {
    c.device = cfg->device;
    if (cfg->max_graphs > 0) c.max_graphs = cfg->max_graphs;
    if (cfg->arena_bytes > 0) c.arena_bytes = cfg->arena_bytes;
    if (cfg->max_v > 0) c.max_v = cfg->max_v;
    if (cfg->max_degree > 0) c.max_degree = cfg->max_degree;
    if (cfg->max_two_hop > 0) c.max_two_hop = cfg->max_two_hop;
    if (cfg->idle_exit_ns > 0) c.idle_exit_ns = cfg->idle_exit_ns;
  }
  if (c.max_graphs > (1 << 24)) return set_error(MBE_ERR_INVALID, "max_graphs above 2^24");
  if ((c.arena_bytes >> kServeBlockShift) > INT32_MAX)
    return set_error(MBE_ERR_INVALID, "arena above 2^31 blocks");
  mbe_server* s = new mbe_server();
  s->device = c.device;
  s->cfg = c;
  if (params) s->prm = *params;
  else mbe_params_default(&s->prm);
  memset(&s->st, 0, sizeof(s->st));
  int rc = allocate(s);
  if (rc) {
    release(s);
    delete s;
    return rc;
  }
  s->loop = std::thread(server_loop, s);
  *out = s;
  return MBE_OK;
}

int mbe_server_submit(mbe_server* s, const int32_t* row_off, const int32_t* col, int32_t nV,
                      int32_t nU, int64_t nE, const mbe_opts* opts, uint64_t* request_id) {
  clear_error();
  if (!s || !request_id) return set_error(MBE_ERR_INVALID, "null argument");
  mbe_opts o;
  if (opts) o = *opts;
  else mbe_opts_default(&o);
  // Host preparation runs in the caller's thread, outside the server lock.
  HostGraph h;
  int rc = build_host_graph(row_off, col, nV, nU, nE, o, &h);
  if (rc) return rc;
  int32_t capL = 1, capS = 1;
  if ((rc = graph_caps(h, &capL, &capS))) return rc;
  auto reject = [&](const char* what, long long got, long long cap) {
    std::lock_guard<std::mutex> lk(s->mu);
    s->st.rejected++;
    return set_error(MBE_ERR_ADMISSION, "%s %lld exceeds the server's %lld", what, got, cap);
  };
  if (h.V_size > s->map_words) return reject("internal V side", h.V_size, s->map_words);
  if (capL > s->capL) return reject("root degree", capL, s->capL);
  if (capS > s->capS) return reject("two-hop multiset", capS, s->capS);

  Request* r = new Request();
  DevGraph& g = r->dg;
  memset(&g, 0, sizeof(g));
  g.nV = h.V_size;
  g.nU = h.U_size;
  g.nE = h.edge_size;
  g.swapped = h.swapped;
  g.root_end = h.V_size;
  g.root_offset = 0;
  g.root_stride = 1;
  g.n_roots = h.V_size;
  if ((rc = apply_tuning(s->prm, &g))) {
    delete r;
    return rc;
  }
  size_t off = align_up(sizeof(ServeGraph), kArrayAlign);
  auto place = [&](size_t bytes) {
    size_t o2 = off;
    off = align_up(off + std::max<size_t>(bytes, 4), kArrayAlign);
    return o2;
  };
  r->o_row_off = place(sizeof(int32_t) * h.row_off.size());
  r->o_col = place(sizeof(int32_t) * h.col.size());
  r->o_rev_off = place(sizeof(int32_t) * h.rev_off.size());
  r->o_rev_col = place(sizeof(int32_t) * h.rev_col.size());
  r->o_ukey = place(sizeof(uint64_t) * (size_t)h.U_size);
  r->o_vkey = place(sizeof(uint64_t) * (size_t)h.V_size);
  r->bytes = align_up(off, kBlock);
  if (r->bytes > (size_t)s->cfg.arena_bytes) {
    const long long need = (long long)r->bytes;
    delete r;
    return reject("graph block bytes", need, s->cfg.arena_bytes);
  }
  r->image.assign(r->bytes, 0);
  auto put = [&](size_t o2, const void* src, size_t bytes) {
    if (bytes) memcpy(r->image.data() + o2, src, bytes);
  };
  put(r->o_row_off, h.row_off.data(), sizeof(int32_t) * h.row_off.size());
  put(r->o_col, h.col.data(), sizeof(int32_t) * h.col.size());
  put(r->o_rev_off, h.rev_off.data(), sizeof(int32_t) * h.rev_off.size());
  put(r->o_rev_col, h.rev_col.data(), sizeof(int32_t) * h.rev_col.size());
  std::vector<uint64_t> uk, vk;
  host_keys(h, &uk, &vk);
  put(r->o_ukey, uk.data(), sizeof(uint64_t) * uk.size());
  put(r->o_vkey, vk.data(), sizeof(uint64_t) * vk.size());
  r->t_submit = now_s();

  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stopping) {
    delete r;
    return set_error(MBE_ERR_INVALID, "server is shutting down");
  }
  if (s->fatal != MBE_OK) {
    delete r;
    return set_error(s->fatal, "server failed earlier: %s", s->fatal_msg.c_str());
  }
  r->id = s->next_id++;
  s->reqs[r->id] = r;
  s->st.submitted++;
  if (g.n_roots == 0) {  // nothing to enumerate
    memset(&r->res, 0, sizeof(r->res));
    s->st.completed++;
    finish(s, r, MBE_OK);
  } else {
    s->waiting.push_back(r);
    s->cv_loop.notify_one();
  }
  *request_id = r->id;
  return MBE_OK;
}

int mbe_server_poll(mbe_server* s, uint64_t request_id, mbe_result* out) {
  clear_error();
  if (!s) return set_error(MBE_ERR_INVALID, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  return take(s, request_id, out);
}

int mbe_server_wait(mbe_server* s, uint64_t request_id, int64_t timeout_ns, mbe_result* out) {
  clear_error();
  if (!s) return set_error(MBE_ERR_INVALID, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  const auto deadline =
      std::chrono::steady_clock::now() + std::chrono::nanoseconds(std::max<int64_t>(timeout_ns, 0));
  while (true) {
    int rc = take(s, request_id, out);
    if (rc != MBE_ERR_AGAIN) return rc;
    if (timeout_ns < 0) s->cv_done.wait(lk);
    else if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout)
      return take(s, request_id, out);
  }
}

int mbe_server_cancel(mbe_server* s, uint64_t request_id) {
  clear_error();
  if (!s) return set_error(MBE_ERR_INVALID, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(request_id);
  if (it == s->reqs.end())
    return set_error(MBE_ERR_NOT_FOUND, "unknown request %llu", (unsigned long long)request_id);
  Request* r = it->second;
  if (r->state != kWaiting)
    return set_error(MBE_ERR_INVALID, "request %llu is already on the GPU or finished",
                     (unsigned long long)request_id);
  r->state = kCancelled;
  // Out of the admission queue now: poll may delete it at once.
  s->waiting.erase(std::remove(s->waiting.begin(), s->waiting.end(), r), s->waiting.end());
  r->image.clear();
  r->image.shrink_to_fit();
  s->st.cancelled++;
  s->cv_done.notify_all();
  return MBE_OK;
}

int mbe_server_get_stats(mbe_server* s, mbe_server_stats* out) {
  clear_error();
  if (!s || !out) return set_error(MBE_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->st;
  out->resident = s->resident;
  out->waiting = (int64_t)s->waiting.size();
  out->arena_used = (int64_t)s->bump;
  out->arena_bytes = s->cfg.arena_bytes;
  out->published = s->published;
  out->collected = s->collected;
  out->launch_running = s->running ? 1 : 0;
  // Device side, read on a stream of its own while a launch may run.
  ServeCtl sc;
  EnumCtl ctl;
  cudaSetDevice(s->device);
  if (cudaMemcpyAsync(&sc, s->d_sctl, sizeof(sc), cudaMemcpyDeviceToHost, s->s_peek) == cudaSuccess &&
      cudaMemcpyAsync(&ctl, s->d_ctl, sizeof(ctl), cudaMemcpyDeviceToHost, s->s_peek) == cudaSuccess &&
      cudaStreamSynchronize(s->s_peek) == cudaSuccess) {
    out->dev_head = sc.arr_head;
    out->dev_tail = sc.arr_tail;
    out->dev_done = sc.done_pos;
    out->dev_pending = ctl.pending;
  }
  return MBE_OK;
}

int mbe_server_debug_request(mbe_server* s, uint64_t request_id, uint64_t out[4]) {
  clear_error();
  if (!s || !out) return set_error(MBE_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(request_id);
  if (it == s->reqs.end() || it->second->state != kResident)
    return set_error(MBE_ERR_INVALID, "request %llu is not on the device",
                     (unsigned long long)request_id);
  ServeGraph hdr;
  cudaSetDevice(s->device);
  if (cudaMemcpyAsync(&hdr, s->d_arena + it->second->arena_off, sizeof(hdr),
                      cudaMemcpyDeviceToHost, s->s_peek) != cudaSuccess ||
      cudaStreamSynchronize(s->s_peek) != cudaSuccess)
    return set_error(MBE_ERR_CUDA, "reading the request's block failed");
  out[0] = hdr.next_root;
  out[1] = hdr.pending;
  out[2] = (uint64_t)hdr.g.n_roots;
  out[3] = it->second->arena_off >> kServeBlockShift;
  return MBE_OK;
}

int mbe_server_destroy(mbe_server* s) {
  clear_error();
  if (!s) return MBE_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
    // Graphs still on the GPU are abandoned: the launch leaves between tasks.
    int32_t one = 1;
    cudaSetDevice(s->device);
    cudaMemcpyAsync(&s->d_sctl->stop, &one, sizeof(one), cudaMemcpyHostToDevice, s->s_copy);
    cudaStreamSynchronize(s->s_copy);
    for (auto& kv : s->reqs)
      if (kv.second->state == kWaiting || kv.second->state == kResident)
        finish(s, kv.second, MBE_ERR_CANCELLED);
    s->waiting.clear();
    s->cv_loop.notify_one();
  }
  if (s->loop.joinable()) s->loop.join();
  release(s);
  delete s;
  return MBE_OK;
}

}  // extern "C"
