// Seeded synthetic bipartite graphs for the benchmark configurations.
//
// Method: Chung-Lu edge sampling.  Expected degrees w_i = c * (i+1)^(-1/(gamma-1)),
// capped at max_deg, with c chosen by bisection so that sum_i min(w_i, cap)
// equals the edge target.  Each edge draws its U end and its V end
// independently in proportion to w (Vose's alias method), duplicates are
// removed, and draws are topped up until the edge target is reached.
// Random numbers come from splitmix64 (Steele, Lea and Flood, "Fast
// splittable pseudorandom number generators", OOPSLA 2014).
//
// Output convention (the .adj contract, preprocess/data_convert.cpp:20-43):
// V rows sorted ascending and deduplicated, V rows of degree 0 dropped, and U
// ids renumbered densely in increasing order of the generated id, so that
// every U id in [0, U_size) has at least one edge.  This keeps every row
// non-empty on both sides, which matters because the reference swaps sides
// under -t and an empty row is undefined behaviour there.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "internal.h"

namespace gmbe {
namespace {

struct SplitMix64 {
  uint64_t s;
  explicit SplitMix64(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
  uint64_t below(uint64_t n) { return (uint64_t)(uniform() * (double)n) % (n ? n : 1); }
};

// Vose's alias table over non-negative weights.
struct Alias {
  std::vector<double> prob;
  std::vector<int32_t> alias;
  explicit Alias(const std::vector<double>& w) {
    size_t n = w.size();
    prob.assign(n, 0.0);
    alias.assign(n, 0);
    double sum = 0;
    for (double x : w) sum += x;
    std::vector<double> p(n);
    std::vector<int32_t> small, large;
    for (size_t i = 0; i < n; ++i) {
      p[i] = w[i] * (double)n / sum;
      (p[i] < 1.0 ? small : large).push_back((int32_t)i);
    }
    while (!small.empty() && !large.empty()) {
      int32_t s = small.back(), l = large.back();
      small.pop_back();
      prob[s] = p[s];
      alias[s] = l;
      p[l] = (p[l] + p[s]) - 1.0;
      if (p[l] < 1.0) {
        large.pop_back();
        small.push_back(l);
      }
    }
    for (int32_t l : large) prob[l] = 1.0;
    for (int32_t s : small) prob[s] = 1.0;
  }
  int32_t draw(SplitMix64& rng) const {
    size_t n = prob.size();
    size_t i = (size_t)rng.below(n);
    return rng.uniform() < prob[i] ? (int32_t)i : alias[i];
  }
};

std::vector<double> power_law_weights(int64_t n, double gamma, int64_t cap, double total) {
  std::vector<double> base(n);
  double alpha = 1.0 / (gamma - 1.0);
  for (int64_t i = 0; i < n; ++i) base[i] = std::pow((double)(i + 1), -alpha);
  double capd = cap > 0 ? (double)cap : 1e300;
  auto sum_at = [&](double c) {
    double s = 0;
    for (double b : base) s += std::min(c * b, capd);
    return s;
  };
  double lo = 0, hi = 1;
  while (sum_at(hi) < total && hi < 1e30) hi *= 2;
  for (int it = 0; it < 200; ++it) {
    double mid = 0.5 * (lo + hi);
    (sum_at(mid) < total ? lo : hi) = mid;
  }
  std::vector<double> w(n);
  for (int64_t i = 0; i < n; ++i) w[i] = std::min(hi * base[i], capd);
  return w;
}

void sort_unique(std::vector<uint64_t>* e) {
  std::sort(e->begin(), e->end());
  e->erase(std::unique(e->begin(), e->end()), e->end());
}

}  // namespace
}  // namespace gmbe

using namespace gmbe;

extern "C" int mbe_gen_chung_lu(const mbe_gen_spec* spec, int32_t** row_off_out, int32_t** col_out,
                                int32_t* nV_out, int32_t* nU_out, int64_t* nE_out) {
  clear_error();
  if (!spec || !row_off_out || !col_out || !nV_out || !nU_out || !nE_out)
    return set_error(MBE_ERR_INVALID, "null argument");
  const mbe_gen_spec& s = *spec;
  if (s.nU <= 0 || s.nV <= 0 || s.n_edges < 0 || s.nU >= INT32_MAX || s.nV >= INT32_MAX ||
      s.gamma_u <= 1.0 || s.gamma_v <= 1.0)
    return set_error(MBE_ERR_INVALID, "bad generator spec");
  if (s.n_blocks > 0 && ((int64_t)s.n_blocks * s.block_u > s.nU || (int64_t)s.n_blocks * s.block_v > s.nV))
    return set_error(MBE_ERR_INVALID, "planted blocks do not fit");
  SplitMix64 rng(s.seed);
  int64_t target = std::min<int64_t>(s.n_edges, s.nU * s.nV);
  // Under a pair-probability cap the graph's density cannot exceed the cap:
  // an edge target above cap * |U| * |V| would be reached only by drawing
  // until nearly every pair is taken (a near-complete block).
  if (s.pair_p_max > 0 && s.pair_p_max < 1)
    target = std::min<int64_t>(target, std::max<int64_t>(1, (int64_t)(s.pair_p_max * (double)s.nU * (double)s.nV)));
  std::vector<double> wu = power_law_weights(s.nU, s.gamma_u, s.max_deg_u, (double)target);
  std::vector<double> wv = power_law_weights(s.nV, s.gamma_v, s.max_deg_v, (double)target);
  Alias au(wu), av(wv);
  // Edge key: v in the high 32 bits so sorted keys are V-major CSR order.
  std::vector<uint64_t> edges;
  edges.reserve((size_t)(target * 1.1) + 1024);
  // Expected multiplicity of pair (u,v) under edge sampling is
  // lambda = w_u w_v / W (W = sum of weights = target); after deduplication
  // P(edge) = 1 - exp(-lambda).  Thinning each draw by min(1, lmax/lambda)
  // caps that probability at pair_p_max.
  const double W = (double)target;
  const double lmax = s.pair_p_max > 0 && s.pair_p_max < 1 ? -std::log(1.0 - s.pair_p_max) : 0.0;
  for (int round = 0; round < 64 && (int64_t)edges.size() < target; ++round) {
    int64_t draws = (round == 0) ? target : (int64_t)((target - (int64_t)edges.size()) * 1.25) + 16;
    for (int64_t k = 0; k < draws; ++k) {
      int32_t u = au.draw(rng), v = av.draw(rng);
      if (lmax > 0) {
        double lam = wu[u] * wv[v] / W;
        if (lam > lmax && rng.uniform() * lam >= lmax) continue;
      }
      edges.push_back(((uint64_t)v << 32) | (uint64_t)u);
    }
    sort_unique(&edges);
  }
  if (s.n_blocks > 0) {
    // Disjoint random vertex sets by partial Fisher-Yates shuffles.
    auto pick = [&](int64_t n, int64_t k) {
      std::vector<int32_t> ids(n);
      for (int64_t i = 0; i < n; ++i) ids[i] = (int32_t)i;
      for (int64_t i = 0; i < k; ++i) {
        int64_t j = i + (int64_t)rng.below((uint64_t)(n - i));
        std::swap(ids[i], ids[j]);
      }
      ids.resize(k);
      return ids;
    };
    std::vector<int32_t> bu = pick(s.nU, (int64_t)s.n_blocks * s.block_u);
    std::vector<int32_t> bv = pick(s.nV, (int64_t)s.n_blocks * s.block_v);
    for (int32_t b = 0; b < s.n_blocks; ++b)
      for (int32_t i = 0; i < s.block_u; ++i)
        for (int32_t j = 0; j < s.block_v; ++j)
          if (rng.uniform() < s.block_p) {
            uint64_t u = (uint64_t)bu[(size_t)b * s.block_u + i];
            uint64_t v = (uint64_t)bv[(size_t)b * s.block_v + j];
            edges.push_back((v << 32) | u);
          }
    sort_unique(&edges);
  }
  // Dense U renumbering (increasing generated id) and V row compaction.
  std::vector<int32_t> umap(s.nU, -1);
  for (uint64_t e : edges) umap[(int64_t)(e & 0xffffffffULL)] = 0;
  int32_t nU = 0;
  for (int64_t u = 0; u < s.nU; ++u)
    if (umap[u] == 0) umap[u] = nU++;
  int64_t nE = (int64_t)edges.size();
  int32_t* col = (int32_t*)malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(nE, 1));
  int32_t* row = (int32_t*)malloc(sizeof(int32_t) * (size_t)(s.nV + 1));
  if (!col || !row) {
    free(col);
    free(row);
    return set_error(MBE_ERR_NOMEM, "out of host memory");
  }
  int32_t nV = 0;
  row[0] = 0;
  int64_t prev_v = -1;
  for (int64_t i = 0; i < nE; ++i) {
    int64_t v = (int64_t)(edges[i] >> 32);
    if (v != prev_v) {
      if (prev_v >= 0) row[++nV] = (int32_t)i;
      prev_v = v;
    }
    col[i] = umap[(int64_t)(edges[i] & 0xffffffffULL)];
  }
  if (prev_v >= 0) row[++nV] = (int32_t)nE;
  *row_off_out = row;
  *col_out = col;
  *nV_out = nV;
  *nU_out = nU;
  *nE_out = nE;
  return MBE_OK;
}

extern "C" int mbe_gen_batch_spec(uint64_t seed, mbe_gen_spec* out) {
  clear_error();
  if (!out) return set_error(MBE_ERR_INVALID, "null argument");
  SplitMix64 rng(seed ^ 0x5bd1e9955bd1e995ULL);
  double lu = std::log(50.0) + rng.uniform() * (std::log(5000.0) - std::log(50.0));
  double lr = std::log(0.5) + rng.uniform() * (std::log(4.0) - std::log(0.5));
  double avg = 3.0 + rng.uniform() * 27.0;
  memset(out, 0, sizeof(*out));
  out->nU = (int64_t)std::llround(std::exp(lu));
  out->nV = std::max<int64_t>(2, (int64_t)std::llround(std::exp(lu) * std::exp(lr)));
  out->n_edges = (int64_t)std::llround(avg * (double)out->nU);
  out->gamma_u = out->gamma_v = 2.2;
  // No degree cap is named for this distribution; Chung-Lu's own condition
  // for edge probabilities to stay below 1 is w_max <= sqrt(total weight).
  const int64_t cap = std::max<int64_t>(2, (int64_t)std::sqrt((double)out->n_edges));
  out->max_deg_u = std::min<int64_t>(cap, out->nV);
  out->max_deg_v = std::min<int64_t>(cap, out->nU);
  out->seed = seed;
  out->pair_p_max = 0.1;
  return MBE_OK;
}

extern "C" int mbe_write_adj(const char* path, const int32_t* row_off, const int32_t* col,
                             int32_t nV) {
  clear_error();
  if (!path || (nV > 0 && (!row_off || !col))) return set_error(MBE_ERR_INVALID, "null argument");
  FILE* fp = fopen(path, "wb");
  if (!fp) return set_error(MBE_ERR_IO, "cannot write %s", path);
  std::vector<char> line;
  char num[16];
  for (int32_t v = 0; v < nV; ++v) {
    line.clear();
    for (int32_t i = row_off[v]; i < row_off[v + 1]; ++i) {
      int n = snprintf(num, sizeof(num), i == row_off[v] ? "%d" : " %d", col[i]);
      line.insert(line.end(), num, num + n);
    }
    line.push_back('\n');
    if (fwrite(line.data(), 1, line.size(), fp) != line.size()) {
      fclose(fp);
      return set_error(MBE_ERR_IO, "short write to %s", path);
    }
  }
  fclose(fp);
  return MBE_OK;
}

extern "C" int mbe_write_graph(const char* path, const int32_t* row_off, const int32_t* col,
                               int32_t nV) {
  clear_error();
  if (!path || (nV > 0 && (!row_off || !col))) return set_error(MBE_ERR_INVALID, "null argument");
  int32_t umax = -1;
  for (int64_t i = 0; nV > 0 && i < (int64_t)row_off[nV]; ++i) umax = std::max(umax, col[i]);
  FILE* fp = fopen(path, "wb");
  if (!fp) return set_error(MBE_ERR_IO, "cannot write %s", path);
  bool ok = fprintf(fp, "%d %d\n", nV, umax + 1) > 0;
  for (int32_t v = 0; ok && v < nV; ++v)
    for (int32_t i = row_off[v]; ok && i < row_off[v + 1]; ++i)
      ok = fprintf(fp, "%d %d\n", v, col[i]) > 0;
  if (fclose(fp) != 0) ok = false;
  return ok ? MBE_OK : set_error(MBE_ERR_IO, "short write to %s", path);
}

extern "C" int mbe_read_adj(const char* path, int32_t** row_off_out, int32_t** col_out,
                            int32_t* nV, int32_t* nU, int64_t* nE) {
  clear_error();
  if (!path || !row_off_out || !col_out || !nV || !nU || !nE)
    return set_error(MBE_ERR_INVALID, "null argument");
  std::vector<int32_t> ro, co;
  int32_t u = 0;
  int rc = read_adj_file(path, &ro, &co, &u);
  if (rc) return rc;
  int32_t* r = (int32_t*)malloc(sizeof(int32_t) * ro.size());
  int32_t* c = (int32_t*)malloc(sizeof(int32_t) * std::max<size_t>(co.size(), 1));
  if (!r || !c) {
    free(r);
    free(c);
    return set_error(MBE_ERR_NOMEM, "out of host memory");
  }
  memcpy(r, ro.data(), sizeof(int32_t) * ro.size());
  if (!co.empty()) memcpy(c, co.data(), sizeof(int32_t) * co.size());
  *row_off_out = r;
  *col_out = c;
  *nV = (int32_t)ro.size() - 1;
  *nU = u;
  *nE = (int64_t)co.size();
  return MBE_OK;
}

extern "C" void mbe_free(void* p) { free(p); }
