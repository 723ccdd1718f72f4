// Enumeration without any device allocation.
//
// Some callers cannot call cudaMalloc: code running inside a framework that
// owns all device memory through its own allocator, code recorded into a
// CUDA graph, or a host process where an allocation at an arbitrary point
// would break a memory budget fixed up front.  mbe_enumerate allocates its
// workspace on first use; this entry point instead takes every working buffer
// it needs from one file-scope __device__ pool of kNoAllocPoolBytes (64 MiB).
// That pool is part of the library's device image: every GPU that loads the
// library holds it until the process exits, whether or not this entry point
// is used.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "engine.h"

namespace {

constexpr size_t kNoAllocPoolBytes = size_t(64) << 20;  // 64 MiB
constexpr int32_t kNoAllocQueueCap = 4096;
constexpr int kNoAllocMaxDevices = 64;
constexpr int kNoAllocMaxBlocks = 1024;

// The pool.  In host code this name is only a host-side stand-in for the
// device symbol: its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_pool[kNoAllocPoolBytes];

struct PoolAddr {
  unsigned char* ptr = nullptr;
};
PoolAddr g_pool_addr[kNoAllocMaxDevices];
std::mutex g_pool_mu;

size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

__device__ __forceinline__ uint64_t fmix64_d(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ULL;
  k ^= k >> 33;
  return k;
}

// Hash keys for the identity numbering (vertex ids are the input ids).
__global__ void noalloc_keys(uint64_t* ukey, int32_t nU, uint64_t* vkey, int32_t nV) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)nU + nV;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (i < nU) ukey[i] = fmix64_d((uint64_t)i * 2u);
    else vkey[i - nU] = fmix64_d((uint64_t)(i - nU) * 2u + 1u);
  }
}

// Places the graph descriptor and the root prefix in the pool and zeroes the
// per-graph results (a kernel, so no host copy is involved).
__global__ void noalloc_init(const gmbe::DevGraph dg, gmbe::DevGraph* d_graph, long long* prefix,
                             unsigned long long* gres) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    *d_graph = dg;
    prefix[0] = 0;
    prefix[1] = dg.n_roots;
    gres[0] = gres[1] = gres[2] = 0;
  }
}

__global__ void noalloc_finish(const gmbe::EnumCtl* ctl, const unsigned long long* gres,
                               unsigned long long* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    out[0] = gres[0];
    out[1] = gres[1];
    out[2] = gres[2];
    out[3] = (unsigned long long)(long long)ctl->status;
  }
}

}  // namespace

using namespace gmbe;

// No counterpart in the reference (see include/mbe.h).
extern "C" int mbe_enumerate_device_noalloc(const int32_t* d_row_off, const int32_t* d_col,
                                            int32_t nV, const int32_t* d_rev_off,
                                            const int32_t* d_rev_col, int32_t nU, int64_t nE,
                                            int64_t max_two_hop, const mbe_params* params,
                                            unsigned long long* d_out, void* stream) {
  clear_error();
  if (!d_row_off || !d_col || !d_rev_off || !d_rev_col || !d_out || nV < 0 || nU < 0 || nE < 0)
    return set_error(MBE_ERR_INVALID, "null or negative argument");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  mbe_params prm;
  if (params) prm = *params;
  else mbe_params_default(&prm);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_error(MBE_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return set_error(MBE_ERR_INVALID, "device %d", dev);

  // One-time set-up per device, with that device current: the pool's device
  // address.  This happens inside the first call on each device, which must
  // therefore come before any stream capture.
  unsigned char* pool = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (!g_pool_addr[dev].ptr) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_pool);
      if (e != cudaSuccess)
        return set_error(MBE_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
      g_pool_addr[dev].ptr = static_cast<unsigned char*>(p);
    }
    pool = g_pool_addr[dev].ptr;
  }

  // Per-warp capacities.  Without a host copy of the graph the bounds are
  // the graph-wide ones: |L| <= nU, the two-hop multiset of a root <= nE
  // (or the caller's tighter max_two_hop), the candidate set <= nV.
  int64_t capS64 = max_two_hop > 0 ? std::min<int64_t>(max_two_hop, std::max<int64_t>(nE, 1))
                                    : std::max<int64_t>(nE, 1);
  if (capS64 > INT32_MAX / 2) return set_error(MBE_ERR_CAPACITY, "graph too large for the no-allocation pool");
  int32_t capS = (int32_t)std::max<int64_t>(capS64, 1);
  int32_t capL = std::max(nU, 1);
  int32_t capC = std::max<int32_t>(1, std::min<int32_t>(nV, capS));
  if (capC >= (1 << 24))
    return set_error(MBE_ERR_CAPACITY, "graph too large for the no-allocation pool");
  ScratchLayout sl = make_layout(nV, capC, capL, capS);
  sl.seen_words = 0;  // first touches by global atomics: this launch uses no dynamic shared memory

  // Pool partition: control block, split ring, per-block timing, hash keys,
  // then as many 16-warp blocks of per-warp scratch as fit.
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off = round_up(off + bytes, 256);
    return o;
  };
  const size_t o_ctl = take(sizeof(EnumCtl));
  const size_t o_graph = take(sizeof(DevGraph));
  const size_t o_prefix = take(2 * sizeof(long long));
  const size_t o_gres = take(3 * sizeof(unsigned long long));
  const size_t o_qt = take(sizeof(Task) * kNoAllocQueueCap);
  const size_t o_qs = take(sizeof(unsigned long long) * kNoAllocQueueCap);
  const size_t o_exit = take(2 * sizeof(unsigned long long) * kNoAllocMaxBlocks);
  const size_t o_uk = take(sizeof(uint64_t) * (size_t)std::max(nU, 1));
  const size_t o_vk = take(sizeof(uint64_t) * (size_t)std::max(nV, 1));
  const size_t o_scr = off;
  if (o_scr >= kNoAllocPoolBytes)
    return set_error(MBE_ERR_CAPACITY,
                     "no-allocation pool (%zu bytes) cannot hold the hash keys of %d + %d vertices",
                     kNoAllocPoolBytes, nU, nV);
  const size_t per_block = (size_t)sl.words_per_warp * sizeof(int32_t) * kEnumWarps;
  int fit_blocks = (int)std::min<size_t>((kNoAllocPoolBytes - o_scr) / per_block, kNoAllocMaxBlocks);
  if (fit_blocks < 1)
    return set_error(MBE_ERR_CAPACITY,
                     "graph needs %zu bytes of scratch per %d-warp block; the no-allocation pool "
                     "holds %zu bytes in total (use mbe_enumerate for graphs this large)",
                     per_block, kEnumWarps, kNoAllocPoolBytes);
  int sms = 0, occ = 0;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess ||
      (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, mbe_enum_kernel, kEnumThreads, 0)) !=
          cudaSuccess)
    return set_error(MBE_ERR_CUDA, "device query: %s", cudaGetErrorString(e));
  int blocks = std::min(fit_blocks, std::max(1, sms * occ));
  if (prm.blocks > 0) blocks = std::min(blocks, prm.blocks);
  const int warps = blocks * kEnumWarps;

  EnumCtl* ctl = reinterpret_cast<EnumCtl*>(pool + o_ctl);
  DevGraph* d_graph = reinterpret_cast<DevGraph*>(pool + o_graph);
  long long* d_prefix = reinterpret_cast<long long*>(pool + o_prefix);
  unsigned long long* d_gres = reinterpret_cast<unsigned long long*>(pool + o_gres);
  Task* q_tasks = reinterpret_cast<Task*>(pool + o_qt);
  unsigned long long* q_seq = reinterpret_cast<unsigned long long*>(pool + o_qs);
  unsigned long long* exit_ns = reinterpret_cast<unsigned long long*>(pool + o_exit);
  uint64_t* ukey = reinterpret_cast<uint64_t*>(pool + o_uk);
  uint64_t* vkey = reinterpret_cast<uint64_t*>(pool + o_vk);
  int32_t* scratch = reinterpret_cast<int32_t*>(pool + o_scr);

  // The pool keeps the previous call's contents: zero what must start at
  // zero (control block, ring slot tags, every warp's dense count map and
  // first-touch bitmap).
  if ((e = cudaMemsetAsync(ctl, 0, sizeof(EnumCtl), st)) != cudaSuccess ||
      (e = cudaMemsetAsync(q_seq, 0, sizeof(unsigned long long) * kNoAllocQueueCap, st)) !=
          cudaSuccess ||
      (e = cudaMemset2DAsync(scratch, (size_t)sl.words_per_warp * sizeof(int32_t), 0,
                             (size_t)sl.zero_words * sizeof(int32_t), (size_t)warps, st)) !=
          cudaSuccess)
    return set_error(MBE_ERR_CUDA, "clearing the pool: %s", cudaGetErrorString(e));
  noalloc_keys<<<std::max(1, std::min(1024, (nU + nV + 255) / 256)), 256, 0, st>>>(ukey, nU, vkey,
                                                                                  nV);

  DevGraph dg;
  memset(&dg, 0, sizeof(dg));
  dg.nV = nV;
  dg.nU = nU;
  dg.nE = nE;
  dg.row_off = d_row_off;
  dg.col = d_col;
  dg.rev_off = d_rev_off;
  dg.rev_col = d_rev_col;
  dg.ukey = ukey;
  dg.vkey = vkey;
  dg.swapped = 0;
  dg.root_end = nV;
  dg.root_offset = 0;
  dg.root_stride = 1;
  dg.n_roots = nV;
  mbe_params tune = prm;
  tune.direct_max_c = 1 << 30;  // bitmap tier straight from set-up whenever |L| allows
  int rc = apply_tuning(tune, &dg);
  if (rc) return rc;
  EnumParams ep;
  memset(&ep, 0, sizeof(ep));
  ep.prune = prm.prune;
  ep.n_graphs = 1;
  ep.queue_cap = kNoAllocQueueCap;
  ep.slot_spin_limit = 20000000;
  ep.idle_ns_limit = prm.wait_limit_ns > 0 ? prm.wait_limit_ns : 600LL * 1000000000LL;
  ep.time_limit_ns = prm.time_limit_ns > 0 ? prm.time_limit_ns : 0;
  ep.record_exit = 0;
  SlotPool none;
  memset(&none, 0, sizeof(none));
  none.slots = nullptr;
  none.bits = nullptr;
  none.nslot = 0;  // no sub-problem export out of the static pool
  ep.vertex_split = 1;
  noalloc_init<<<1, 32, 0, st>>>(dg, d_graph, d_prefix, d_gres);
  mbe_enum_kernel<<<blocks, kEnumThreads, 0, st>>>(d_graph, d_prefix, d_gres, ep, sl, ctl, q_tasks,
                                                   q_seq, none, scratch, exit_ns);
  noalloc_finish<<<1, 32, 0, st>>>(ctl, d_gres, d_out);
  if ((e = cudaGetLastError()) != cudaSuccess)
    return set_error(MBE_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
  return MBE_OK;
}
