// Graph build on the device (mbe_graph_build_on_device): the work of
// CSRBiGraph::Read after parsing (src/BiGraph.cu:13-92, 217-277) -- validation,
// the -t side swap, the -o 0/1/2 row ordering, both CSRs -- plus the hash keys
// and the per-warp capacities, on the GPU from the uploaded .adj-shaped CSR.
//
// The -o order is the host build's exactly: rows by size, then by content
// (lexicographic, as the reference's comparator, src/BiGraph.cu:75-85), then
// by original id, so a graph built here has the same internal ids, hence the
// same roots in every root range and shard, as one built on the host.
//
// Sorting uses CUB (header-only, shipped with the CUDA toolkit): a merge sort
// of row ids under that comparator for the order, stable radix sorts for the
// transposes; the other steps are the kernels below.  The row offsets are
// checked on the host (O(nV)) before any kernel indexes through them; the
// entries (O(nE)) are checked on the device before anything is built from them.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <numeric>
#include <vector>

#include "engine.h"
#include "internal.h"
#include "mbe.h"

namespace gmbe {
namespace {

#define DCK(call)                                                                          \
  do {                                                                                     \
    cudaError_t _e = (call);                                                               \
    if (_e != cudaSuccess) {                                                               \
      rc = set_error(MBE_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(_e));               \
      goto done;                                                                           \
    }                                                                                      \
  } while (0)

constexpr int kThreads = 256;

int blocks_for(int64_t threads) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((threads + kThreads - 1) / kThreads, 1 << 16));
}

__device__ __forceinline__ uint64_t fmix64_d(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ULL;
  k ^= k >> 33;
  return k;
}

// One warp per row: the row of every entry, the largest id, and the .adj
// entry checks.  flags[0] = largest id; flags[1] = first error seen: 1 an id
// out of range, 2 a row not strictly ascending.
__global__ void k_scan_rows(const int32_t* off, const int32_t* col, int32_t n, int32_t nU,
                            int32_t* row_of, int32_t* flags) {
  const int lane = threadIdx.x & 31;
  for (int v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n;
       v += (gridDim.x * blockDim.x) >> 5) {
    const int32_t b = off[v], e = off[v + 1];
    int32_t mx = -1, bad = 0;
    for (int32_t j = b + lane; j < e; j += 32) {
      const int32_t u = col[j];
      row_of[j] = v;
      mx = max(mx, u);
      if (u < 0 || u == INT32_MAX || (nU > 0 && u >= nU)) bad = 1;
      else if (j + 1 < e && col[j + 1] <= u) bad = max(bad, 2);
    }
    mx = __reduce_max_sync(0xffffffffu, mx);
    bad = __reduce_max_sync(0xffffffffu, bad);
    if (lane == 0) {
      atomicMax(&flags[0], mx);
      if (bad) atomicCAS(&flags[1], 0, bad);
    }
  }
}

__global__ void k_histogram(const int32_t* keys, int64_t n, int32_t* count) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&count[keys[e]], 1);
}

// One warp per row: the row of every entry (entries stored in row order).
__global__ void k_rows_of(const int32_t* off, int32_t n, int32_t* row_of) {
  const int lane = threadIdx.x & 31;
  for (int v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n;
       v += (gridDim.x * blockDim.x) >> 5)
    for (int32_t j = off[v] + lane; j < off[v + 1]; j += 32) row_of[j] = v;
}

__global__ void k_iota(int32_t n, int32_t* ident) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    ident[v] = v;
}

// The row order of -o 1 (ascending size) and -o 2 (descending): equal sizes
// compare by content, lexicographically ascending, then by row id (the row's
// original id, which makes the order total).
struct RowOrder {
  const int32_t* off;
  const int32_t* adj;
  int32_t descending;
  __device__ bool operator()(const int32_t& a, const int32_t& b) const {
    const int32_t sa = off[a + 1] - off[a], sb = off[b + 1] - off[b];
    if (sa != sb) return descending ? sa > sb : sa < sb;
    const int32_t* pa = adj + off[a];
    const int32_t* pb = adj + off[b];
    for (int32_t i = 0; i < sa; ++i)
      if (pa[i] != pb[i]) return pa[i] < pb[i];
    return a < b;
  }
};

__global__ void k_permuted_degrees(const int32_t* off, const int32_t* perm, int32_t n, int32_t* out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = off[perm[i] + 1] - off[perm[i]];
}

// New row i = old row perm[i]: one warp per row.
__global__ void k_gather_rows(const int32_t* off, const int32_t* adj, const int32_t* perm,
                              const int32_t* new_off, int32_t n, int32_t* new_adj) {
  const int lane = threadIdx.x & 31;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n;
       i += (gridDim.x * blockDim.x) >> 5) {
    const int32_t src = perm[i], b = off[src], len = off[src + 1] - b, o = new_off[i];
    for (int32_t j = lane; j < len; j += 32) new_adj[o + j] = adj[b + j];
  }
}

// Hash keys of the internal sides, over original ids and original sides
// (the same keys as the host build's).
__global__ void k_keys(const int32_t* v_orig, int32_t nV, int32_t nU, int32_t swapped,
                       uint64_t* vkey, uint64_t* ukey) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < max(nV, nU); i += gridDim.x * blockDim.x) {
    if (i < nV) vkey[i] = fmix64_d((uint64_t)v_orig[i] * 2u + (swapped ? 0u : 1u));
    if (i < nU) ukey[i] = fmix64_d((uint64_t)i * 2u + (swapped ? 1u : 0u));
  }
}

// Capacities and degree maxima: out[0] = max row degree, out[1] = max over
// rows v of sum_{u in N(v)} d(u) (the two-hop multiset a root's set-up walks),
// out[2] = max U degree.  One warp per row.
__global__ void k_caps(const int32_t* off, const int32_t* adj, const int32_t* uoff, int32_t nV,
                       int32_t nU, unsigned long long* out) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int v = warp; v < nV; v += nw) {
    unsigned long long s = 0;
    for (int32_t j = off[v] + lane; j < off[v + 1]; j += 32) {
      const int32_t u = adj[j];
      s += (unsigned long long)(uoff[u + 1] - uoff[u]);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
      atomicMax(&out[0], (unsigned long long)(off[v + 1] - off[v]));
      atomicMax(&out[1], s);
    }
  }
  for (int u = warp * 32 + lane; u < nU; u += nw * 32)
    atomicMax(&out[2], (unsigned long long)(uoff[u + 1] - uoff[u]));
}

// Transpose of a CSR whose entries are ids < n_dst with row_of[e] the row of
// entry e: a stable radix sort of (id, row) pairs lists every destination
// row's sources in ascending order; a histogram and a scan give the offsets.
int transpose_dev(const int32_t* d_adj, const int32_t* d_row_of, int64_t nE, int32_t n_dst,
                  int32_t* d_toff, int32_t* d_tadj) {
  int rc = MBE_OK;
  int32_t *keys_out = nullptr, *cnt = nullptr;
  void* tmp = nullptr;
  size_t sort_bytes = 0, scan_bytes = 0;
  int end_bit = 1;
  while (end_bit < 31 && (1ll << end_bit) < (long long)n_dst) ++end_bit;
  DCK(cudaMalloc((void**)&keys_out, sizeof(int32_t) * std::max<int64_t>(nE, 1)));
  DCK(cudaMalloc((void**)&cnt, sizeof(int32_t) * ((size_t)n_dst + 1)));
  DCK(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, d_adj, keys_out, d_row_of, d_tadj,
                                      (int)nE, 0, end_bit));
  DCK(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, cnt, d_toff, n_dst + 1));
  DCK(cudaMalloc(&tmp, std::max<size_t>(std::max(sort_bytes, scan_bytes), 1)));
  DCK(cub::DeviceRadixSort::SortPairs(tmp, sort_bytes, d_adj, keys_out, d_row_of, d_tadj, (int)nE,
                                      0, end_bit));
  DCK(cudaMemset(cnt, 0, sizeof(int32_t) * ((size_t)n_dst + 1)));
  k_histogram<<<blocks_for(nE), kThreads>>>(d_adj, nE, cnt);
  DCK(cudaGetLastError());
  DCK(cub::DeviceScan::ExclusiveSum(tmp, scan_bytes, cnt, d_toff, n_dst + 1));
done:
  cudaFree(keys_out);
  cudaFree(cnt);
  cudaFree(tmp);
  return rc;
}

// Row offsets of an .adj-shaped CSR, checked on the host before any kernel
// reads through them (the messages of validate_adj_csr).
int check_offsets(const int32_t* row_off, int32_t nV, int64_t nE) {
  if (row_off[0] != 0) return set_error(MBE_ERR_FORMAT, "row_off[0] must be 0");
  if ((int64_t)row_off[nV] != nE)
    return set_error(MBE_ERR_FORMAT, "row_off[nV]=%d does not match nE=%lld", row_off[nV],
                     (long long)nE);
  for (int32_t v = 0; v < nV; ++v) {
    if (row_off[v + 1] < row_off[v])
      return set_error(MBE_ERR_FORMAT, "row %d: decreasing offsets", v);
    if (row_off[v + 1] == row_off[v])
      return set_error(MBE_ERR_FORMAT, "row %d is empty (.adj lines must be non-empty)", v);
  }
  return MBE_OK;
}

}  // namespace

int device_build_graph(mbe_graph* g, const int32_t* row_off, const int32_t* col, int32_t nV,
                       int32_t nU, int64_t nE) {
  const mbe_opts& o = g->opts;
  if (nV <= 0 || nE <= 0 || !row_off || !col)
    return set_error(MBE_ERR_INVALID, "invalid CSR arguments (nV=%d nE=%lld)", nV, (long long)nE);
  if (nE > INT32_MAX) return set_error(MBE_ERR_FORMAT, "more than 2^31-1 edges");
  int rc = check_offsets(row_off, nV, nE);
  if (rc) return rc;
  int32_t *d_ro = nullptr, *d_co = nullptr, *d_rowof = nullptr, *d_uoff = nullptr,
          *d_uadj = nullptr,
          *d_perm = nullptr, *d_pdeg = nullptr, *d_flags = nullptr;
  unsigned long long* d_caps = nullptr;
  void* tmp = nullptr;
  int32_t flags[2] = {-1, 0};
  unsigned long long caps[3] = {0, 0, 0};
  const int32_t *voff = nullptr, *vadj = nullptr;
  int32_t iV = 0, iU = 0;
  bool swap = false;
  size_t sort_bytes = 0, scan_bytes = 0;
  HostGraph& h = g->h;
  DCK(cudaSetDevice(g->device));
  DCK(cudaMalloc((void**)&d_ro, sizeof(int32_t) * ((size_t)nV + 1)));
  DCK(cudaMalloc((void**)&d_co, sizeof(int32_t) * nE));
  DCK(cudaMalloc((void**)&d_rowof, sizeof(int32_t) * nE));
  DCK(cudaMalloc((void**)&d_flags, sizeof(flags)));
  DCK(cudaMemcpy(d_ro, row_off, sizeof(int32_t) * ((size_t)nV + 1), cudaMemcpyHostToDevice));
  DCK(cudaMemcpy(d_co, col, sizeof(int32_t) * nE, cudaMemcpyHostToDevice));
  DCK(cudaMemcpy(d_flags, flags, sizeof(flags), cudaMemcpyHostToDevice));
  k_scan_rows<<<blocks_for((int64_t)nV * 32), kThreads>>>(d_ro, d_co, nV, nU, d_rowof, d_flags);
  DCK(cudaGetLastError());
  DCK(cudaMemcpy(flags, d_flags, sizeof(flags), cudaMemcpyDeviceToHost));
  if (flags[1] == 1) {
    rc = set_error(MBE_ERR_FORMAT, "U id out of range (nU %d)", nU);
    goto done;
  }
  if (flags[1] == 2) {
    rc = set_error(MBE_ERR_FORMAT, "U ids of a row not strictly ascending");
    goto done;
  }
  if (nU <= 0) nU = flags[0] + 1;
  // U -> V adjacency of the input.
  DCK(cudaMalloc((void**)&d_uoff, sizeof(int32_t) * ((size_t)nU + 1)));
  DCK(cudaMalloc((void**)&d_uadj, sizeof(int32_t) * nE));
  if ((rc = transpose_dev(d_co, d_rowof, nE, nU, d_uoff, d_uadj))) goto done;
  // -t (src/BiGraph.cu:67-73): 1 makes V the smaller side, 2 the larger.
  swap = (o.uvtrans == 1 && nU < nV) || (o.uvtrans == 2 && nU > nV);
  voff = swap ? d_uoff : d_ro;
  vadj = swap ? d_uadj : d_co;
  iV = swap ? nU : nV;
  iU = swap ? nV : nU;
  // -o: 0 keeps the input order; 1 sorts rows by degree ascending; every
  // other value descending (the reference comparator's reading under -f).
  DCK(cudaMalloc((void**)&d_perm, sizeof(int32_t) * iV));
  DCK(cudaMalloc((void**)&d_pdeg, sizeof(int32_t) * ((size_t)iV + 1)));
  DCK(cudaMalloc((void**)&d_caps, sizeof(caps)));
  k_iota<<<blocks_for(iV), kThreads>>>(iV, d_perm);
  DCK(cudaGetLastError());
  {
    const RowOrder cmp{voff, vadj, o.order == 1 ? 0 : 1};
    DCK(cub::DeviceMergeSort::SortKeys(nullptr, sort_bytes, d_perm, (int64_t)iV, cmp));
    DCK(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, d_pdeg, d_pdeg, iV + 1));
    DCK(cudaMalloc(&tmp, std::max<size_t>(std::max(sort_bytes, scan_bytes), 1)));
    if (o.order != 0) DCK(cub::DeviceMergeSort::SortKeys(tmp, sort_bytes, d_perm, (int64_t)iV, cmp));
  }
  k_permuted_degrees<<<blocks_for(iV), kThreads>>>(voff, d_perm, iV, d_pdeg);
  DCK(cudaGetLastError());
  DCK(cudaMemset(d_pdeg + iV, 0, sizeof(int32_t)));
  DCK(cudaMalloc((void**)&g->d_row_off, sizeof(int32_t) * ((size_t)iV + 1)));
  DCK(cub::DeviceScan::ExclusiveSum(tmp, scan_bytes, d_pdeg, g->d_row_off, iV + 1));
  DCK(cudaMalloc((void**)&g->d_col, sizeof(int32_t) * nE));
  k_gather_rows<<<blocks_for((int64_t)iV * 32), kThreads>>>(voff, vadj, d_perm, g->d_row_off, iV,
                                                            g->d_col);
  DCK(cudaGetLastError());
  // Internal U -> V lists, over internal V ids.
  k_rows_of<<<blocks_for((int64_t)iV * 32), kThreads>>>(g->d_row_off, iV, d_rowof);
  DCK(cudaGetLastError());
  DCK(cudaMalloc((void**)&g->d_rev_off, sizeof(int32_t) * ((size_t)iU + 1)));
  DCK(cudaMalloc((void**)&g->d_rev_col, sizeof(int32_t) * nE));
  if ((rc = transpose_dev(g->d_col, d_rowof, nE, iU, g->d_rev_off, g->d_rev_col))) goto done;
  DCK(cudaMalloc((void**)&g->d_vkey, sizeof(uint64_t) * iV));
  DCK(cudaMalloc((void**)&g->d_ukey, sizeof(uint64_t) * iU));
  k_keys<<<blocks_for(std::max(iV, iU)), kThreads>>>(d_perm, iV, iU, swap ? 1 : 0, g->d_vkey,
                                                     g->d_ukey);
  DCK(cudaGetLastError());
  DCK(cudaMemset(d_caps, 0, sizeof(caps)));
  k_caps<<<blocks_for((int64_t)iV * 32), kThreads>>>(g->d_row_off, g->d_col, g->d_rev_off, iV, iU,
                                                     d_caps);
  DCK(cudaGetLastError());
  DCK(cudaMemcpy(caps, d_caps, sizeof(caps), cudaMemcpyDeviceToHost));
  if (caps[1] > (unsigned long long)(INT32_MAX / 2)) {
    rc = set_error(MBE_ERR_CAPACITY, "two-hop multiset of a root exceeds 2^30 entries");
    goto done;
  }
  h.U_size = iU;
  h.V_size = iV;
  h.edge_size = nE;
  h.swapped = swap ? 1 : 0;
  h.V_degree = (int32_t)caps[0];
  h.U_degree = (int32_t)caps[2];
  h.U_2degree = h.V_2degree = 0;
  h.v_orig.resize(iV);
  DCK(cudaMemcpy(h.v_orig.data(), d_perm, sizeof(int32_t) * iV, cudaMemcpyDeviceToHost));
  h.u_orig.resize(iU);
  std::iota(h.u_orig.begin(), h.u_orig.end(), 0);
  g->capS = (int32_t)std::max<unsigned long long>(caps[1], 1);
  g->capL = (int32_t)std::max<unsigned long long>(caps[0], 1);
  g->device_built = true;
done:
  cudaFree(d_ro);
  cudaFree(d_co);
  cudaFree(d_rowof);
  cudaFree(d_uoff);
  cudaFree(d_uadj);
  cudaFree(d_perm);
  cudaFree(d_pdeg);
  cudaFree(d_flags);
  cudaFree(d_caps);
  cudaFree(tmp);
  return rc;
}

int ensure_host_csr(mbe_graph* g) {
  if (!g->device_built || !g->h.row_off.empty()) return MBE_OK;
  HostGraph& h = g->h;
  h.row_off.resize((size_t)h.V_size + 1);
  h.col.resize((size_t)h.edge_size);
  h.rev_off.resize((size_t)h.U_size + 1);
  h.rev_col.resize((size_t)h.edge_size);
  cudaError_t e = cudaSetDevice(g->device);
  if (e == cudaSuccess)
    e = cudaMemcpy(h.row_off.data(), g->d_row_off, sizeof(int32_t) * h.row_off.size(),
                   cudaMemcpyDeviceToHost);
  if (e == cudaSuccess)
    e = cudaMemcpy(h.col.data(), g->d_col, sizeof(int32_t) * h.col.size(), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess)
    e = cudaMemcpy(h.rev_off.data(), g->d_rev_off, sizeof(int32_t) * h.rev_off.size(),
                   cudaMemcpyDeviceToHost);
  if (e == cudaSuccess)
    e = cudaMemcpy(h.rev_col.data(), g->d_rev_col, sizeof(int32_t) * h.rev_col.size(),
                   cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    h.row_off.clear();
    return set_error(MBE_ERR_CUDA, "fetching the graph: %s", cudaGetErrorString(e));
  }
  return MBE_OK;
}

}  // namespace gmbe
