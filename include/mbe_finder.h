// mbe_finder.h -- the reference's C++ surface over the C ABI of mbe.h.
//
// Same class names, constructor arguments and member meaning as the
// reference, so a caller of the reference compiles against this header:
//   struct Option                 src/BiGraph.h:13-22
//   struct CSRBiGraph             src/BiGraph.h:23-38  (Read, CopyToGpu, Reset)
//   class BicliqueFinder          src/BicliqueFinder.h:18-30 (Execute, PrintResult)
//   class IterFinderGpu6          src/IterFinderGpu.h:77-90 (bound_height, bound_size)
//   class IterFinderGpu           src/IterFinderGpu.h:18-30 (-s 0 entry; runs the same engine)
// Differences, by design:
//   - maximal_nodes_ is unsigned long long (the reference's int wraps past 2^31);
//     PrintResult keeps the reference's text ("maximal nodes:%llu").
//   - Errors do not exit the process: Read() leaves an empty graph and
//     Execute() leaves status() != 0; last_error() gives the message.
//   - The finder never copies the graph again: CSRBiGraph::Read already holds
//     the device copy (the reference copies it in the finder constructor,
//     src/IterFinderGpu.cu:181-201, 1056-1085).
#pragma once

#include <cstdio>
#include <string>

#include "mbe.h"

struct Option {
  int uvtrans;
  int order;
  int fast_mode;
  Option() : uvtrans(0), order(1), fast_mode(0) {}
};

struct CSRBiGraph {
  CSRBiGraph();
  ~CSRBiGraph();
  CSRBiGraph(const CSRBiGraph&) = delete;
  CSRBiGraph& operator=(const CSRBiGraph&) = delete;
  // Parses the .adj file and uploads it (reference Read + CopyToGpu).  Prints
  // the reference's "Graph:..." line.  Returns an MBE status.
  int Read(const char* filename, Option opt);
  // Builds from an in-memory .adj-shaped CSR (V rows of U ids).
  int FromCSR(const int32_t* row_off, const int32_t* col, int32_t nV, int32_t nU, int64_t nE,
              Option opt);
  void Reset();
  int U_size, V_size, edge_size, U_degree, V_degree, U_2degree, V_2degree;
  bool device_graph;
  mbe_graph* handle;
};

class BicliqueFinder {
 public:
  BicliqueFinder() = delete;
  explicit BicliqueFinder(CSRBiGraph* graph_in);
  virtual ~BicliqueFinder() {}
  virtual void Execute() = 0;
  void PrintResult(char* fn = nullptr);
  unsigned long long maximal_nodes() const { return maximal_nodes_; }
  double exe_time() const { return exe_time_; }

 protected:
  CSRBiGraph* graph_;
  unsigned long long maximal_nodes_;
  double exe_time_, start_time_;
};

class IterFinderGpu6 : public BicliqueFinder {
 public:
  IterFinderGpu6() = delete;
  IterFinderGpu6(CSRBiGraph* graph_in, int bound_height = 20, int bound_size = 1500);
  virtual void Execute();
  // Extras not in the reference's class.
  const mbe_result& result() const { return result_; }
  int status() const { return status_; }
  std::string last_error() const { return error_; }
  mbe_params& params() { return params_; }

 protected:
  mbe_params params_;
  mbe_result result_;
  int status_;
  std::string error_;
};

// -s 0 / -s 1 of the reference select its ablation kernels (GMBE-WARP,
// GMBE-BLOCK); here they run the same engine with task splitting disabled.
class IterFinderGpu : public IterFinderGpu6 {
 public:
  explicit IterFinderGpu(CSRBiGraph* graph_in);
};

class IterFinderGpu2 : public IterFinderGpu6 {
 public:
  explicit IterFinderGpu2(CSRBiGraph* graph_in);
};
