// The reference's C++ classes (CSRBiGraph, BicliqueFinder, IterFinderGpu6)
// implemented over the C ABI.
#include "mbe_finder.h"

#include <sys/time.h>

#include <cstring>

namespace {
double wall_s() {
  struct timeval tv;
  gettimeofday(&tv, nullptr);
  return (double)tv.tv_sec + (double)tv.tv_usec * 1e-6;
}
}  // namespace

CSRBiGraph::CSRBiGraph()
    : U_size(0), V_size(0), edge_size(0), U_degree(0), V_degree(0), U_2degree(0), V_2degree(0),
      device_graph(false), handle(nullptr) {}

CSRBiGraph::~CSRBiGraph() { Reset(); }

static void fill_info(CSRBiGraph* g) {
  mbe_graph_info info;
  mbe_graph_get_info(g->handle, &info);
  g->U_size = info.U_size;
  g->V_size = info.V_size;
  g->edge_size = (int)info.edge_size;
  g->U_degree = info.U_degree;
  g->V_degree = info.V_degree;
  g->U_2degree = info.U_2degree;
  g->V_2degree = info.V_2degree;
  g->device_graph = true;
}

int CSRBiGraph::Read(const char* filename, Option opt) {
  Reset();
  mbe_opts o;
  mbe_opts_default(&o);
  o.uvtrans = opt.uvtrans;
  o.order = opt.order;
  o.fast_mode = opt.fast_mode;
  int rc = mbe_graph_from_adj(filename, &o, &handle);
  if (rc != MBE_OK) {
    // Reference: "Can't open file <name>" on stderr, graph left empty (src/BiGraph.cu:15-18).
    fprintf(stderr, "%s\n", mbe_last_error_string());
    handle = nullptr;
    return rc;
  }
  fill_info(this);
  // Reference output line (src/BiGraph.cu:212-215, 247-248).
  printf("Graph:%s ", filename);
  if (!opt.fast_mode) {
    printf("|U|:%8d |V|:%8d |E|:%8d ", U_size, V_size, edge_size);
    printf("d(U):%8d d2(U):%8d ", U_degree, U_2degree);
    printf("d(V):%8d d2(V):%8d\n", V_degree, V_2degree);
  } else {
    printf("|U|:%8d |V|:%8d |E|:%8d\n", U_size, V_size, edge_size);
  }
  return MBE_OK;
}

int CSRBiGraph::FromCSR(const int32_t* row_off, const int32_t* col, int32_t nV, int32_t nU,
                        int64_t nE, Option opt) {
  Reset();
  mbe_opts o;
  mbe_opts_default(&o);
  o.uvtrans = opt.uvtrans;
  o.order = opt.order;
  o.fast_mode = opt.fast_mode;
  int rc = mbe_graph_from_csr(row_off, col, nV, nU, nE, &o, &handle);
  if (rc != MBE_OK) {
    handle = nullptr;
    return rc;
  }
  fill_info(this);
  return MBE_OK;
}

void CSRBiGraph::Reset() {
  if (handle) mbe_graph_free(handle);
  handle = nullptr;
  U_size = V_size = edge_size = 0;
  U_degree = V_degree = U_2degree = V_2degree = 0;
  device_graph = false;
}

BicliqueFinder::BicliqueFinder(CSRBiGraph* graph_in)
    : graph_(graph_in), maximal_nodes_(0), exe_time_(0), start_time_(0) {}

void BicliqueFinder::PrintResult(char* fn) {
  // Same text as src/BicliqueFinder.cu:9-16.
  FILE* fp = (fn == nullptr || strlen(fn) == 0) ? stdout : fopen(fn, "a+");
  if (!fp) return;
  if (fp != stdout) fseek(fp, 0, SEEK_END);
  fprintf(fp, "Total processing time: %lf seconds\n", exe_time_);
  fprintf(fp, "maximal nodes:%llu\n", maximal_nodes_);
  fprintf(fp, "\n");
  if (fp != stdout) fclose(fp);
}

IterFinderGpu6::IterFinderGpu6(CSRBiGraph* graph_in, int bound_height, int bound_size)
    : BicliqueFinder(graph_in), status_(0) {
  mbe_params_default(&params_);
  params_.bound_height = bound_height;
  params_.bound_size = bound_size;
  memset(&result_, 0, sizeof(result_));
}

void IterFinderGpu6::Execute() {
  start_time_ = wall_s();
  if (!graph_ || !graph_->handle) {
    status_ = MBE_ERR_INVALID;
    error_ = "graph not loaded";
    exe_time_ = wall_s() - start_time_;
    return;
  }
  status_ = mbe_enumerate(graph_->handle, &params_, &result_);
  if (status_ != MBE_OK) error_ = mbe_last_error_string();
  maximal_nodes_ = result_.count;
  exe_time_ = wall_s() - start_time_;
}

IterFinderGpu::IterFinderGpu(CSRBiGraph* graph_in) : IterFinderGpu6(graph_in, 1 << 30, 1 << 30) {}

IterFinderGpu2::IterFinderGpu2(CSRBiGraph* graph_in) : IterFinderGpu6(graph_in, 1 << 30, 1 << 30) {}
