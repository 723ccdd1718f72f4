// Internal declarations shared by the host-side translation units of libgmbe.
#pragma once

#include <cstdarg>
#include <cstdint>
#include <string>
#include <vector>

#include "mbe.h"

namespace gmbe {

// Records `msg` as the calling thread's last error and returns `code`.
int set_error(int code, const char* fmt, ...);
void clear_error();

// Host graph in the engine's internal numbering (after -t swap and -o order).
//   row_off/col      : V -> U adjacency (V rows, ascending U ids)       (reference row_offset/column_indices)
//   rev_off/rev_col  : U -> V adjacency (U rows, ascending internal V)   (reference rev_row_offset/rev_column_indices)
//   v_orig[v]        : original id of internal V vertex v (a line number, or a U id when swapped)
//   u_orig[u]        : original id of internal U vertex u
struct HostGraph {
  int32_t U_size = 0, V_size = 0;
  int64_t edge_size = 0;
  int32_t U_degree = 0, V_degree = 0, U_2degree = 0, V_2degree = 0;
  int32_t swapped = 0;
  std::vector<int32_t> row_off, col, rev_off, rev_col, v_orig, u_orig;
};

// Validates an .adj-shaped CSR (rows strictly ascending, non-empty, ids in range).
int validate_adj_csr(const int32_t* row_off, const int32_t* col, int32_t nV, int32_t nU, int64_t nE);

// Applies the -t swap and -o ordering and builds both CSRs on the host
// (restates src/BiGraph.cu:67-92 and 217-277).
int build_host_graph(const int32_t* row_off, const int32_t* col, int32_t nV, int32_t nU,
                     int64_t nE, const mbe_opts& opts, HostGraph* out);

// Reads .adj into CSR vectors; nU = max id + 1.
int read_adj_file(const char* path, std::vector<int32_t>* row_off, std::vector<int32_t>* col,
                  int32_t* nU);

}  // namespace gmbe
