// Host-side graph ingest: .adj parsing, validation, the -t side swap, the -o
// row ordering and the two CSRs.  Restates the behaviour of CSRBiGraph::Read
// (src/BiGraph.cu:13-278); the data layout it produces is the one the device
// engine consumes (internal V rows = enumeration roots).
#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>

#include "internal.h"

namespace gmbe {

thread_local std::string g_last_error;

int set_error(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

void clear_error() { g_last_error.clear(); }

int validate_adj_csr(const int32_t* row_off, const int32_t* col, int32_t nV, int32_t nU,
                     int64_t nE) {
  if (nV < 0 || nE < 0 || (nV > 0 && (!row_off || (nE > 0 && !col))))
    return set_error(MBE_ERR_INVALID, "invalid CSR arguments (nV=%d nE=%lld)", nV, (long long)nE);
  if (nV > 0 && row_off[0] != 0) return set_error(MBE_ERR_FORMAT, "row_off[0] must be 0");
  if (nV > 0 && (int64_t)row_off[nV] != nE)
    return set_error(MBE_ERR_FORMAT, "row_off[nV]=%d does not match nE=%lld", row_off[nV],
                     (long long)nE);
  for (int32_t v = 0; v < nV; ++v) {
    int32_t b = row_off[v], e = row_off[v + 1];
    if (e < b) return set_error(MBE_ERR_FORMAT, "row %d: decreasing offsets", v);
    // An empty row makes the reference read vertices[-1]
    // (src/IterFinderGpu.cu:682 via 794); it is rejected here.
    if (e == b) return set_error(MBE_ERR_FORMAT, "row %d is empty (.adj lines must be non-empty)", v);
    for (int32_t i = b; i < e; ++i) {
      int32_t u = col[i];
      if (u < 0 || u == INT32_MAX || (nU > 0 && u >= nU))
        return set_error(MBE_ERR_FORMAT, "row %d: U id %d out of range", v, u);
      // Binary searches over rows rely on strictly ascending ids
      // (src/GpuUtil.cuh:71-83).
      if (i > b && col[i - 1] >= u)
        return set_error(MBE_ERR_FORMAT, "row %d: ids not strictly ascending (%d then %d)", v,
                         col[i - 1], u);
    }
  }
  return MBE_OK;
}

int read_adj_file(const char* path, std::vector<int32_t>* row_off, std::vector<int32_t>* col,
                  int32_t* nU) {
  FILE* fp = fopen(path, "rb");
  if (!fp) return set_error(MBE_ERR_IO, "Can't open file %s", path);
  row_off->clear();
  col->clear();
  row_off->push_back(0);
  int64_t maxid = -1;
  std::vector<char> buf(1 << 22);
  int64_t cur = -1;  // token being parsed, -1 = none
  bool line_has_data = false;
  int64_t line_no = 0;
  auto end_line = [&](void) {
    row_off->push_back((int32_t)col->size());
    line_has_data = false;
    ++line_no;
  };
  size_t n;
  bool bad = false;
  char bad_ch = 0;
  while ((n = fread(buf.data(), 1, buf.size(), fp)) > 0 && !bad) {
    for (size_t i = 0; i < n; ++i) {
      char c = buf[i];
      if (c >= '0' && c <= '9') {
        cur = (cur < 0 ? 0 : cur) * 10 + (c - '0');
        if (cur >= INT32_MAX) { bad = true; bad_ch = '#'; break; }
        line_has_data = true;
      } else {
        if (cur >= 0) {
          col->push_back((int32_t)cur);
          if (cur > maxid) maxid = cur;
          cur = -1;
        }
        if (c == '\n') {
          end_line();
        } else if (c == ' ' || c == '\t' || c == '\r') {
        } else {
          bad = true;
          bad_ch = c;
          break;
        }
      }
    }
  }
  fclose(fp);
  if (bad) {
    if (bad_ch == '#') return set_error(MBE_ERR_FORMAT, "%s line %lld: id >= 2^31-1", path, (long long)line_no + 1);
    return set_error(MBE_ERR_FORMAT, "%s line %lld: unexpected character 0x%02x", path,
                     (long long)line_no + 1, (unsigned char)bad_ch);
  }
  if (cur >= 0) {
    col->push_back((int32_t)cur);
    if (cur > maxid) maxid = cur;
  }
  // A final line without '\n' still counts (std::getline semantics).
  if (line_has_data || (int64_t)col->size() > (int64_t)row_off->back()) end_line();
  if (col->size() > (size_t)INT32_MAX)
    return set_error(MBE_ERR_FORMAT, "%s: more than 2^31-1 edges", path);
  *nU = (int32_t)(maxid + 1);
  return MBE_OK;
}

// Two-hop degree statistics of the non-fast path (src/BiGraph.cu:39-65):
// max over vertices of |N(N(x))| - 1.
static int32_t max_two_hop(const std::vector<int32_t>& off, const std::vector<int32_t>& adj,
                           const std::vector<int32_t>& roff, const std::vector<int32_t>& radj,
                           int32_t n_self) {
  std::vector<int32_t> mark(n_self, -1);
  int32_t best = 0;
  for (int32_t x = 0; x + 1 < (int32_t)off.size(); ++x) {
    int32_t cnt = 0;
    for (int32_t i = off[x]; i < off[x + 1]; ++i) {
      int32_t y = adj[i];
      for (int32_t j = roff[y]; j < roff[y + 1]; ++j) {
        int32_t z = radj[j];
        if (mark[z] != x) {
          mark[z] = x;
          ++cnt;
        }
      }
    }
    best = std::max(best, cnt - 1);
  }
  return best;
}

// Builds the transpose of a CSR whose rows are [0,n_rows) and columns [0,n_cols).
static void transpose(const std::vector<int32_t>& off, const std::vector<int32_t>& adj,
                      int32_t n_rows, int32_t n_cols, std::vector<int32_t>* toff,
                      std::vector<int32_t>* tadj) {
  toff->assign((size_t)n_cols + 1, 0);
  for (int32_t x : adj) (*toff)[x + 1]++;
  for (int32_t i = 0; i < n_cols; ++i) (*toff)[i + 1] += (*toff)[i];
  tadj->assign(adj.size(), 0);
  std::vector<int32_t> fill(toff->begin(), toff->end() - 1);
  for (int32_t r = 0; r < n_rows; ++r)
    for (int32_t i = off[r]; i < off[r + 1]; ++i) (*tadj)[fill[adj[i]]++] = r;
}

// Two-hop peeling order of -o 3 (src/BiGraph.cu:93-210): vertices are bucketed
// by their exact two-hop degree and repeatedly the vertex of smallest remaining
// two-hop degree is taken, lowering the degree of its not-yet-taken two-hop
// neighbours (bucket peeling as in Batagelj-Zaversnik k-core ordering).
static std::vector<int32_t> two_hop_peel_order(const std::vector<int32_t>& off,
                                               const std::vector<int32_t>& adj,
                                               const std::vector<int32_t>& roff,
                                               const std::vector<int32_t>& radj, int32_t n) {
  std::vector<int32_t> deg(n, 0), mark(n, -1);
  for (int32_t x = 0; x < n; ++x) {
    int32_t c = 0;
    for (int32_t i = off[x]; i < off[x + 1]; ++i)
      for (int32_t j = roff[adj[i]]; j < roff[adj[i] + 1]; ++j) {
        int32_t z = radj[j];
        if (z != x && mark[z] != x) {
          mark[z] = x;
          ++c;
        }
      }
    deg[x] = c;
  }
  int32_t maxd = 0;
  for (int32_t d : deg) maxd = std::max(maxd, d);
  std::vector<int32_t> start((size_t)maxd + 2, 0);
  for (int32_t d : deg) start[d + 1]++;
  for (int32_t d = 0; d <= maxd; ++d) start[d + 1] += start[d];
  std::vector<int32_t> order(n), pos(n), next(start.begin(), start.end() - 1);
  for (int32_t x = 0; x < n; ++x) {
    pos[x] = next[deg[x]]++;
    order[pos[x]] = x;
  }
  std::vector<int32_t> bstart(start.begin(), start.end() - 1);
  std::fill(mark.begin(), mark.end(), -1);
  for (int32_t k = 0; k < n; ++k) {
    int32_t x = order[k];
    for (int32_t i = off[x]; i < off[x + 1]; ++i)
      for (int32_t j = roff[adj[i]]; j < roff[adj[i] + 1]; ++j) {
        int32_t y = radj[j];
        if (mark[y] == x) continue;
        mark[y] = x;
        if (deg[y] > deg[x]) {
          // Move y to the front of its bucket, then shrink its degree.
          int32_t dy = deg[y], py = pos[y], pw = bstart[dy], w = order[pw];
          if (y != w) {
            pos[y] = pw;
            order[py] = w;
            pos[w] = py;
            order[pw] = y;
          }
          bstart[dy]++;
          deg[y]--;
        }
      }
  }
  return order;
}

int build_host_graph(const int32_t* row_off, const int32_t* col, int32_t nV, int32_t nU,
                     int64_t nE, const mbe_opts& opts, HostGraph* g) {
  int32_t maxid = -1;
  for (int64_t i = 0; i < nE; ++i) maxid = std::max(maxid, col[i]);
  if (nU <= 0) nU = maxid + 1;
  if (maxid >= nU) return set_error(MBE_ERR_FORMAT, "U id %d >= nU %d", maxid, nU);
  int rc = validate_adj_csr(row_off, col, nV, nU, nE);
  if (rc) return rc;
  if (nE > INT32_MAX) return set_error(MBE_ERR_FORMAT, "more than 2^31-1 edges");

  std::vector<int32_t> voff(row_off, row_off + nV + 1), vadj(col, col + nE);
  std::vector<int32_t> uoff, uadj;
  transpose(voff, vadj, nV, nU, &uoff, &uadj);
  std::vector<int32_t> vorig(nV), uorig(nU);
  std::iota(vorig.begin(), vorig.end(), 0);
  std::iota(uorig.begin(), uorig.end(), 0);

  g->U_degree = g->V_degree = g->U_2degree = g->V_2degree = 0;
  for (int32_t v = 0; v < nV; ++v) g->V_degree = std::max(g->V_degree, voff[v + 1] - voff[v]);
  for (int32_t u = 0; u < nU; ++u) g->U_degree = std::max(g->U_degree, uoff[u + 1] - uoff[u]);
  if (!opts.fast_mode) {
    g->U_2degree = max_two_hop(uoff, uadj, voff, vadj, nU);
    g->V_2degree = max_two_hop(voff, vadj, uoff, uadj, nV);
  }
  // -t: 1 makes V the smaller side, 2 the larger (src/BiGraph.cu:67-73, 217-227).
  bool swap = (opts.uvtrans == 1 && nU < nV) || (opts.uvtrans == 2 && nU > nV);
  if (swap) {
    std::swap(nU, nV);
    std::swap(voff, uoff);
    std::swap(vadj, uadj);
    std::swap(vorig, uorig);
    std::swap(g->U_degree, g->V_degree);
    std::swap(g->U_2degree, g->V_2degree);
  }
  g->swapped = swap ? 1 : 0;

  // -o: reorder V rows.  1/2: by size (asc/desc), ties lexicographic
  // ascending (src/BiGraph.cu:75-85, 228-238); identical rows are ordered by
  // original id so the result is deterministic.  Under fast_mode the
  // reference's comparator sends every order other than 1 to "descending",
  // so -o 3 -f behaves as -o 2.  Without fast_mode, -o 3 is two-hop peeling.
  std::vector<int32_t> perm(nV);
  std::iota(perm.begin(), perm.end(), 0);
  if (opts.order == 3 && !opts.fast_mode) {
    perm = two_hop_peel_order(voff, vadj, uoff, uadj, nV);
  } else if (opts.order != 0) {
    bool asc = opts.order == 1;
    std::sort(perm.begin(), perm.end(), [&](int32_t a, int32_t b) {
      int32_t sa = voff[a + 1] - voff[a], sb = voff[b + 1] - voff[b];
      if (sa != sb) return asc ? sa < sb : sa > sb;
      const int32_t* pa = &vadj[voff[a]];
      const int32_t* pb = &vadj[voff[b]];
      for (int32_t i = 0; i < sa; ++i)
        if (pa[i] != pb[i]) return pa[i] < pb[i];
      return vorig[a] < vorig[b];
    });
  }
  g->U_size = nU;
  g->V_size = nV;
  g->edge_size = nE;
  g->row_off.assign((size_t)nV + 1, 0);
  g->col.resize(nE);
  g->v_orig.resize(nV);
  for (int32_t i = 0; i < nV; ++i) {
    int32_t src = perm[i];
    int32_t len = voff[src + 1] - voff[src];
    g->row_off[i + 1] = g->row_off[i] + len;
    std::copy(vadj.begin() + voff[src], vadj.begin() + voff[src + 1], g->col.begin() + g->row_off[i]);
    g->v_orig[i] = vorig[src];
  }
  g->u_orig = uorig;
  transpose(g->row_off, g->col, nV, nU, &g->rev_off, &g->rev_col);
  return MBE_OK;
}

}  // namespace gmbe

extern "C" const char* mbe_last_error_string(void) { return gmbe::g_last_error.c_str(); }
