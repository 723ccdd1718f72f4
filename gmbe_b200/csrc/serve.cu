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
//
// Preparation: submit checks the request against the server's capacities
// from the raw CSR (sizes and degrees only, O(edges)) and copies it; a pool of
// preparation threads then builds the -t/-o graph, its hash keys and the
// arena image, so a client that submits many graphs is not held up behind
// each one's sort and transposes.
//
// Emission (mbe_server_set_emit): the launch writes each biclique's L side,
// tagged with the graph's arena block, into a host-mapped ring; the server
// thread drains it while the launch runs, decodes each record against the
// request's prepared graph (kept for this) and hands the biclique to the
// callback.  A graph's completion record carries the ring position past all
// of its records, and its result is released only once the drain has passed
// that position.  The ring restarts from position 0 with every launch, after
// the launch's last records have been drained.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <set>
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

enum ReqState { kPreparing, kWaiting, kResident, kDone, kFailed, kCancelled };

struct Request {
  uint64_t id = 0;
  ReqState state = kPreparing;
  // The submitted CSR, until a preparation thread has built the image.
  std::vector<int32_t> in_off, in_col;
  int32_t in_nV = 0, in_nU = 0;
  mbe_opts opts;
  bool held = false;    // a preparation thread works on it (outside the lock)
  bool orphan = false;  // forgotten while held: the preparation thread deletes it
  std::string msg;      // why it failed, when it failed alone
  std::shared_ptr<const HostGraph> hg;  // the prepared graph, kept to decode emitted records
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
  std::deque<Request*> preparing;  // submitted, not yet taken by a preparation thread
  std::set<uint64_t> prep_ids;     // ids submitted and not yet prepared (queued or held)
  std::deque<Request*> waiting;    // prepared, ascending id
  std::unordered_map<uint64_t, Request*> reqs;
  uint64_t next_id = 1;
  uint64_t published = 0, collected = 0;
  int64_t resident = 0;
  bool stopping = false;
  int fatal = MBE_OK;
  std::string fatal_msg;
  mbe_server_stats st;
  std::thread loop;
  std::condition_variable cv_prep;
  bool prep_stop = false;
  std::vector<std::thread> prep;
  // Emission (all under mu, drained by the server thread only).
  mbe_server_emit_fn emit_fn = nullptr;
  void* emit_user = nullptr;
  int32_t* h_ring = nullptr;         // host-mapped ring of records [|L|, block, L ids]
  int32_t* d_ring = nullptr;
  unsigned long long* h_read = nullptr;  // words consumed, read by the launch
  unsigned long long* d_read = nullptr;
  long long ring_cap = 0;
  unsigned long long ring_pos = 0;   // words taken from the ring in this launch
  unsigned long long ring_done = 0;  // words whose bicliques the callback has had
  struct EmitGraph {
    uint64_t request;
    std::shared_ptr<const HostGraph> hg;
  };
  std::unordered_map<uint32_t, EmitGraph> emit_graphs;  // arena block -> its request
  struct Finishing {  // completed on the device, records still in the ring
    uint64_t request;
    uint32_t blk;
    unsigned long long emit_end, count, hash, non_maximal;
  };
  std::vector<Finishing> finishing;
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
  if (s->h_ring) cudaFreeHost(s->h_ring);
  if (s->h_read) cudaFreeHost(s->h_read);
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
  s->sl = make_layout(s->map_words, s->capC, s->capL, s->capS);
  int rc = enum_blocks_per_sm(false, enum_smem_bytes(s->sl), &occ);
  if (rc) return rc;
  s->blocks = s->prm.blocks > 0 ? std::min(s->prm.blocks, dev_sms * occ) : dev_sms * occ;
  const int warps = s->blocks * kEnumWarps;
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
    if (r->state == kPreparing || r->state == kWaiting || r->state == kResident) finish(s, r, rc);
  }
  s->waiting.clear();
  s->preparing.clear();
  s->prep_ids.clear();
  s->resident = 0;
  s->finishing.clear();
  s->emit_graphs.clear();
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
  if (s->emit_fn) s->emit_graphs[blk] = mbe_server::EmitGraph{r->id, std::move(r->hg)};
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

// Releases a request's result (caller holds mu).
void complete(mbe_server* s, uint64_t id, unsigned long long count, unsigned long long hash,
              unsigned long long non_maximal) {
  auto it = s->reqs.find(id);
  if (it == s->reqs.end() || it->second->state != kResident) return;
  Request* r = it->second;
  memset(&r->res, 0, sizeof(r->res));
  r->res.count = count;
  r->res.set_hash = hash;
  r->res.non_maximal = non_maximal;
  r->res.enum_seconds = now_s() - r->t_submit;
  s->st.completed++;
  finish(s, r, MBE_OK);
}

// Completions whose records have all been handed to the callback (all of
// them when `all`: the launch has ended and its ring is drained).
void release_finished(mbe_server* s, bool all) {
  auto keep = s->finishing.begin();
  for (auto it = s->finishing.begin(); it != s->finishing.end(); ++it) {
    if (all || it->emit_end <= s->ring_done) {
      complete(s, it->request, it->count, it->hash, it->non_maximal);
      s->emit_graphs.erase(it->blk);
    } else {
      *keep++ = *it;
    }
  }
  s->finishing.erase(keep, s->finishing.end());
}

// Takes every committed record off the ring and hands its biclique to the
// callback, with the lock released while decoding and calling (caller holds
// mu through `lk`; only the server thread drains).  True if any was taken.
bool drain_emission(mbe_server* s, std::unique_lock<std::mutex>& lk) {
  struct Rec {
    uint64_t request;
    std::shared_ptr<const HostGraph> hg;
    std::vector<int32_t> L;
  };
  std::vector<Rec> batch;
  volatile int32_t* ring = s->h_ring;
  const unsigned long long cap = (unsigned long long)s->ring_cap;
  const unsigned long long start = s->ring_pos;
  // At most one ring's worth per call: the lock is held while records are
  // taken, and a launch may refill the ring as fast as it is emptied.
  while (s->ring_pos - start < cap) {
    const int32_t len = ring[s->ring_pos % cap];
    if (len <= 0) break;
    const uint32_t blk = (uint32_t)ring[(s->ring_pos + 1) % cap];
    Rec rec;
    rec.L.resize((size_t)len);
    for (int32_t i = 0; i < len; ++i) rec.L[i] = ring[(s->ring_pos + 2 + i) % cap];
    for (int32_t i = 0; i < len + 2; ++i) ring[(s->ring_pos + i) % cap] = 0;
    s->ring_pos += (unsigned long long)len + 2;
    *(volatile unsigned long long*)s->h_read = s->ring_pos;
    auto it = s->emit_graphs.find(blk);
    if (it != s->emit_graphs.end()) {
      rec.request = it->second.request;
      rec.hg = it->second.hg;
      batch.push_back(std::move(rec));
    }
  }
  if (!batch.empty()) {
    lk.unlock();
    std::vector<int32_t> us, vs, R, tmp;
    for (Rec& b : batch) {
      decode_biclique(*b.hg, b.L, &us, &vs, R, tmp);
      s->emit_fn(b.request, us.data(), (int32_t)us.size(), vs.data(), (int32_t)vs.size(),
                 s->emit_user);
    }
    lk.lock();
  }
  s->ring_done = s->ring_pos;
  return s->ring_pos != start;
}

// Completion records, in the order the device handed out their positions
// (caller holds mu).  True if any was taken.
bool collect_completions(mbe_server* s) {
  bool any = false;
  while (true) {
    volatile ServeDone* d = s->h_done + (s->collected % (uint64_t)s->done_cap);
    if (d->seq != s->collected + 1) break;
    const uint64_t id = d->request;
    auto it = s->reqs.find(id);
    if (it != s->reqs.end() && it->second->state == kResident) {
      if (s->emit_fn) {
        // Released once the drain has passed the graph's records.
        s->finishing.push_back(mbe_server::Finishing{
            id, (uint32_t)(it->second->arena_off >> kServeBlockShift), d->emit_end, d->count,
            d->hash, d->non_maximal});
      } else {
        complete(s, id, d->count, d->hash, d->non_maximal);
      }
    }
    s->collected++;
    s->resident--;
    any = true;
  }
  return any;
}

void server_loop(mbe_server* s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    bool progress = false;
    if (s->emit_fn && s->fatal == MBE_OK) {
      progress |= drain_emission(s, lk);
      release_finished(s, false);
    }
    progress |= collect_completions(s);
    if (s->emit_fn) release_finished(s, false);
    // A launch that ended.
    if (s->running && cudaEventQuery(s->ev_run) == cudaSuccess) {
      s->running = false;
      EnumCtl ctl;
      cudaError_t e = cudaMemcpy(&ctl, s->d_ctl, sizeof(ctl), cudaMemcpyDeviceToHost);
      if (e == cudaSuccess && ctl.status == 0 && s->emit_fn) {
        // Completions written just before the end, then every record of the
        // launch (all committed now); the ring restarts with the next launch.
        collect_completions(s);
        while (s->ring_pos < ctl.emit_pos && drain_emission(s, lk)) {
        }
        if (s->ring_pos == ctl.emit_pos) {
          release_finished(s, true);
          s->ring_pos = s->ring_done = 0;
          *(volatile unsigned long long*)s->h_read = 0;
        } else if (!s->stopping) {
          s->fatal = MBE_ERR_CUDA;
          s->fatal_msg = "emission ring: records reserved but never written";
          fail_all(s, s->fatal);
        }
      }
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
    // Admission, first come first served: not past a request submitted
    // earlier that is still being prepared.
    while (!s->waiting.empty() && !s->stopping && s->fatal == MBE_OK) {
      Request* r = s->waiting.front();
      if (!s->prep_ids.empty() && *s->prep_ids.begin() < r->id) break;
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
  if (r->state == kPreparing || r->state == kWaiting || r->state == kResident)
    return MBE_ERR_AGAIN;
  int rc;
  if (r->state == kDone) {
    if (out) *out = r->res;
    rc = MBE_OK;
  } else if (r->state == kCancelled) {
    rc = set_error(MBE_ERR_CANCELLED, "request %llu was cancelled", (unsigned long long)id);
  } else {
    rc = set_error(r->rc, "request %llu failed: %s", (unsigned long long)id,
                   r->msg.empty() ? s->fatal_msg.c_str() : r->msg.c_str());
  }
  s->reqs.erase(it);
  if (r->held) r->orphan = true;  // its preparation thread deletes it
  else delete r;
  return rc;
}

// The server-wide capacities a request must fit, from the raw CSR: the
// internal V side after -t, its largest degree and its largest two-hop
// multiset sum_{y in N(x)} d(y).  None depends on the -o row order, so these
// equal graph_caps() of the built graph.  Also sizes the arena block.
struct Fit {
  int32_t V, U, capL, swapped;
  int64_t capS;
  size_t o_row_off, o_col, o_rev_off, o_rev_col, o_ukey, o_vkey, bytes;
};

int fit_of(const int32_t* row_off, const int32_t* col, int32_t nV, int32_t* nU, int64_t nE,
           const mbe_opts& o, Fit* f) {
  int32_t maxid = -1;
  for (int64_t i = 0; i < nE; ++i) maxid = std::max(maxid, col[i]);
  if (*nU <= 0) *nU = maxid + 1;
  if (maxid >= *nU) return set_error(MBE_ERR_FORMAT, "U id %d >= nU %d", maxid, *nU);
  int rc = validate_adj_csr(row_off, col, nV, *nU, nE);
  if (rc) return rc;
  if (nE > INT32_MAX) return set_error(MBE_ERR_FORMAT, "more than 2^31-1 edges");
  const int32_t n_u = *nU;
  std::vector<int32_t> dcol(n_u, 0);
  for (int64_t i = 0; i < nE; ++i) dcol[col[i]]++;
  const bool swap = (o.uvtrans == 1 && n_u < nV) || (o.uvtrans == 2 && n_u > nV);
  int64_t capS = 0;
  int32_t capL = 0;
  if (!swap) {
    for (int32_t v = 0; v < nV; ++v) {
      int64_t sum = 0;
      for (int32_t i = row_off[v]; i < row_off[v + 1]; ++i) sum += dcol[col[i]];
      capS = std::max(capS, sum);
      capL = std::max(capL, row_off[v + 1] - row_off[v]);
    }
  } else {
    std::vector<int64_t> sum(n_u, 0);
    for (int32_t v = 0; v < nV; ++v) {
      const int32_t d = row_off[v + 1] - row_off[v];
      for (int32_t i = row_off[v]; i < row_off[v + 1]; ++i) sum[col[i]] += d;
    }
    for (int32_t u = 0; u < n_u; ++u) {
      capS = std::max(capS, sum[u]);
      capL = std::max(capL, dcol[u]);
    }
  }
  if (capS > INT32_MAX / 2)
    return set_error(MBE_ERR_CAPACITY, "two-hop multiset of a root exceeds 2^30 entries");
  f->swapped = swap ? 1 : 0;
  f->V = swap ? n_u : nV;
  f->U = swap ? nV : n_u;
  f->capL = std::max(capL, 1);
  f->capS = std::max<int64_t>(capS, 1);
  size_t off = align_up(sizeof(ServeGraph), kArrayAlign);
  auto place = [&](size_t bytes) {
    size_t o2 = off;
    off = align_up(off + std::max<size_t>(bytes, 4), kArrayAlign);
    return o2;
  };
  f->o_row_off = place(sizeof(int32_t) * ((size_t)f->V + 1));
  f->o_col = place(sizeof(int32_t) * (size_t)nE);
  f->o_rev_off = place(sizeof(int32_t) * ((size_t)f->U + 1));
  f->o_rev_col = place(sizeof(int32_t) * (size_t)nE);
  f->o_ukey = place(sizeof(uint64_t) * (size_t)f->U);
  f->o_vkey = place(sizeof(uint64_t) * (size_t)f->V);
  f->bytes = align_up(off, kBlock);
  return MBE_OK;
}

// Builds a request's arena image from its submitted CSR (a preparation
// thread, without the lock).  Writes only into `image`, and into `keep` (the
// prepared graph, for decoding emitted records) when it is not null.
int build_image(const Request* r, std::vector<char>* image, HostGraph* keep) {
  HostGraph h;
  int rc = build_host_graph(r->in_off.data(), r->in_col.data(), r->in_nV, r->in_nU,
                            (int64_t)r->in_col.size(), r->opts, &h);
  if (rc) return rc;
  if (h.V_size != r->dg.nV || h.U_size != r->dg.nU || h.swapped != r->dg.swapped)
    return set_error(MBE_ERR_INVALID, "prepared sides differ from the submitted ones");
  image->assign(r->bytes, 0);
  auto put = [&](size_t o2, const void* src, size_t bytes) {
    if (bytes) memcpy(image->data() + o2, src, bytes);
  };
  put(r->o_row_off, h.row_off.data(), sizeof(int32_t) * h.row_off.size());
  put(r->o_col, h.col.data(), sizeof(int32_t) * h.col.size());
  put(r->o_rev_off, h.rev_off.data(), sizeof(int32_t) * h.rev_off.size());
  put(r->o_rev_col, h.rev_col.data(), sizeof(int32_t) * h.rev_col.size());
  std::vector<uint64_t> uk, vk;
  host_keys(h, &uk, &vk);
  put(r->o_ukey, uk.data(), sizeof(uint64_t) * uk.size());
  put(r->o_vkey, vk.data(), sizeof(uint64_t) * vk.size());
  if (keep) *keep = std::move(h);
  return MBE_OK;
}

// A preparation thread: takes submitted requests in order, builds their
// images and queues them for admission in id order.
void prep_loop(mbe_server* s) {
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    s->cv_prep.wait(lk, [&] { return s->prep_stop || !s->preparing.empty(); });
    if (s->prep_stop) break;
    Request* r = s->preparing.front();
    s->preparing.pop_front();
    r->held = true;
    lk.unlock();
    std::vector<char> image;
    std::shared_ptr<HostGraph> hg = s->emit_fn ? std::make_shared<HostGraph>() : nullptr;
    const int rc = build_image(r, &image, hg.get());
    const std::string msg = rc ? std::string(mbe_last_error_string()) : std::string();
    lk.lock();
    r->held = false;
    s->prep_ids.erase(r->id);
    s->cv_loop.notify_one();  // admission may have waited for this one
    std::vector<int32_t>().swap(r->in_off);
    std::vector<int32_t>().swap(r->in_col);
    if (r->orphan) {
      delete r;
      continue;
    }
    if (r->state != kPreparing) continue;  // cancelled or failed meanwhile
    if (rc) {
      r->msg = msg;
      finish(s, r, rc);
      continue;
    }
    r->image = std::move(image);
    r->hg = std::move(hg);
    r->state = kWaiting;
    auto pos = s->waiting.end();
    while (pos != s->waiting.begin() && (*(pos - 1))->id > r->id) --pos;
    s->waiting.insert(pos, r);
    s->cv_loop.notify_one();
  }
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
    if (cfg->prep_threads > 0) c.prep_threads = cfg->prep_threads;
  }
  if (c.prep_threads <= 0)
    c.prep_threads = (int32_t)std::min(8u, std::max(1u, std::thread::hardware_concurrency()));
  if (c.prep_threads > 256) return set_error(MBE_ERR_INVALID, "prep_threads above 256");
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
  for (int32_t i = 0; i < c.prep_threads; ++i) s->prep.emplace_back(prep_loop, s);
  *out = s;
  return MBE_OK;
}

int mbe_server_submit(mbe_server* s, const int32_t* row_off, const int32_t* col, int32_t nV,
                      int32_t nU, int64_t nE, const mbe_opts* opts, uint64_t* request_id) {
  clear_error();
  if (!s || !request_id) return set_error(MBE_ERR_INVALID, "null argument");
  if (nV < 0 || nE < 0 || (nV > 0 && !row_off) || (nE > 0 && !col))
    return set_error(MBE_ERR_INVALID, "invalid CSR arguments (nV=%d nE=%lld)", nV, (long long)nE);
  const double t_submit = now_s();
  mbe_opts o;
  if (opts) o = *opts;
  else mbe_opts_default(&o);
  Fit f;
  int rc = fit_of(row_off, col, nV, &nU, nE, o, &f);
  if (rc) return rc;
  auto reject = [&](const char* what, long long got, long long cap) {
    std::lock_guard<std::mutex> lk(s->mu);
    s->st.rejected++;
    return set_error(MBE_ERR_ADMISSION, "%s %lld exceeds the server's %lld", what, got, cap);
  };
  if (f.V > s->map_words) return reject("internal V side", f.V, s->map_words);
  if (f.capL > s->capL) return reject("root degree", f.capL, s->capL);
  if (f.capS > s->capS) return reject("two-hop multiset", f.capS, s->capS);
  if (f.bytes > (size_t)s->cfg.arena_bytes)
    return reject("graph block bytes", (long long)f.bytes, s->cfg.arena_bytes);

  Request* r = new Request();
  DevGraph& g = r->dg;
  memset(&g, 0, sizeof(g));
  g.nV = f.V;
  g.nU = f.U;
  g.nE = nE;
  g.swapped = f.swapped;
  g.root_end = f.V;
  g.root_offset = 0;
  g.root_stride = 1;
  g.n_roots = f.V;
  if ((rc = apply_tuning(s->prm, &g))) {
    delete r;
    return rc;
  }
  r->o_row_off = f.o_row_off;
  r->o_col = f.o_col;
  r->o_rev_off = f.o_rev_off;
  r->o_rev_col = f.o_rev_col;
  r->o_ukey = f.o_ukey;
  r->o_vkey = f.o_vkey;
  r->bytes = f.bytes;
  r->opts = o;
  r->in_nV = nV;
  r->in_nU = nU;
  r->t_submit = t_submit;
  if (f.V > 0) {
    r->in_off.assign(row_off, row_off + (size_t)nV + 1);
    r->in_col.assign(col, col + nE);
  }

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
    s->preparing.push_back(r);
    s->prep_ids.insert(r->id);
    s->cv_prep.notify_one();
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
  if (r->state != kWaiting && r->state != kPreparing)
    return set_error(MBE_ERR_INVALID, "request %llu is already on the GPU or finished",
                     (unsigned long long)request_id);
  // Out of the queues now: poll may forget it at once (a preparation thread
  // that holds it deletes it once done).
  if (r->state == kPreparing) {
    s->prep_ids.erase(r->id);  // later requests need not wait for it
    s->cv_loop.notify_one();
    if (!r->held) {
      s->preparing.erase(std::remove(s->preparing.begin(), s->preparing.end(), r),
                         s->preparing.end());
      std::vector<int32_t>().swap(r->in_off);
      std::vector<int32_t>().swap(r->in_col);
    }
  }
  r->state = kCancelled;
  s->waiting.erase(std::remove(s->waiting.begin(), s->waiting.end(), r), s->waiting.end());
  r->image.clear();
  r->image.shrink_to_fit();
  s->st.cancelled++;
  s->cv_done.notify_all();
  return MBE_OK;
}

int mbe_server_set_emit(mbe_server* s, int64_t ring_words, mbe_server_emit_fn fn, void* user) {
  clear_error();
  if (!s || !fn || ring_words < 0) return set_error(MBE_ERR_INVALID, "bad argument");
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->emit_fn || s->st.submitted > 0)
    return set_error(MBE_ERR_INVALID, "emission is set once, before the first submit");
  // The ring holds at least one record of the largest L (a root's degree).
  const long long cap =
      std::max<long long>({ring_words > 0 ? ring_words : (long long)1 << 22,
                           (long long)s->capL + 2, 64});
  SCK(cudaSetDevice(s->device));
  int32_t* h_ring = nullptr;
  unsigned long long* h_read = nullptr;
  cudaError_t e = cudaHostAlloc((void**)&h_ring, sizeof(int32_t) * (size_t)cap, cudaHostAllocMapped);
  if (e == cudaSuccess)
    e = cudaHostAlloc((void**)&h_read, sizeof(unsigned long long), cudaHostAllocMapped);
  if (e == cudaSuccess) {
    memset(h_ring, 0, sizeof(int32_t) * (size_t)cap);
    *h_read = 0;
    e = cudaHostGetDevicePointer((void**)&s->d_ring, h_ring, 0);
  }
  if (e == cudaSuccess) e = cudaHostGetDevicePointer((void**)&s->d_read, h_read, 0);
  if (e != cudaSuccess) {
    if (h_ring) cudaFreeHost(h_ring);
    if (h_read) cudaFreeHost(h_read);
    s->d_ring = nullptr;
    s->d_read = nullptr;
    return set_error(MBE_ERR_NOMEM, "emission ring of %lld words: %s", cap, cudaGetErrorString(e));
  }
  s->h_ring = h_ring;
  s->h_read = h_read;
  s->ring_cap = cap;
  s->ep.emit = s->d_ring;
  s->ep.emit_cap = cap;
  s->ep.emit_read = s->d_read;
  s->emit_user = user;
  s->emit_fn = fn;
  return MBE_OK;
}

int mbe_server_get_stats(mbe_server* s, mbe_server_stats* out) {
  clear_error();
  if (!s || !out) return set_error(MBE_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->st;
  out->resident = s->resident;
  out->waiting = (int64_t)(s->waiting.size() + s->prep_ids.size());
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
    // Also ends a wait for room in the emission ring, which looks only at abort.
    if (s->emit_fn)
      cudaMemcpyAsync(&s->d_ctl->abort, &one, sizeof(one), cudaMemcpyHostToDevice, s->s_copy);
    cudaStreamSynchronize(s->s_copy);
    for (auto& kv : s->reqs)
      if (kv.second->state == kPreparing || kv.second->state == kWaiting ||
          kv.second->state == kResident)
        finish(s, kv.second, MBE_ERR_CANCELLED);
    s->waiting.clear();
    s->preparing.clear();
    s->prep_ids.clear();
    s->prep_stop = true;
    s->cv_prep.notify_all();
    s->cv_loop.notify_one();
  }
  for (std::thread& t : s->prep)
    if (t.joinable()) t.join();
  if (s->loop.joinable()) s->loop.join();
  release(s);
  delete s;
  return MBE_OK;
}

}  // extern "C"
