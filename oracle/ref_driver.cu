// Host-only driver for the reference's in-tree CPU enumerators.
//
// TEST INFRASTRUCTURE ONLY: built by oracle/Makefile (target `ref`) against
// the reference's own sources (src/BiGraph.cu, src/BicliqueFinder.cu,
// src/Utility.cu), output into oracle/_ref/.  It reads an .adj file with
// CSRBiGraph::Read (fast mode) and runs MbeaFinder (sel 0, src/BicliqueFinder.cu:20-57)
// or MbeaFinderBitset (sel 1, src/BicliqueFinder.cu:59-197), printing the
// reference's own result lines ("Total processing time", "maximal nodes").
//
// sel 2 times MbeaFinderBitset on root samples, for the benchmark's CPU
// baseline: MbeaFinderBitset::Execute (src/BicliqueFinder.cu:62-73) calls
// biclique_find(N(v), v, 0) once per V vertex v, and the calls are
// independent, so a sample of roots is a sample of its work.  Sample j
// (j = first .. first+count-1) is the roots v = j, j + stride, j + 2 stride,
// ... below max_root (positions in the reference's own internal order after
// -t/-o, from the lowest degree up; a max_root below 1 is that fraction of
// all roots, 0 = every root).  `first` may instead be a comma-separated list
// of sample offsets, run in that order (count is then ignored).  The roots of a sample run on `threads`
// OpenMP threads, one finder object per thread (the finder's only mutable
// state is its counter).  One line per sample:
//   sample <j> roots <n> count <bicliques> seconds <wall time of the sample>
//
// usage: ref_mbea <file.adj> <sel 0|1> [uvtrans] [order]
//        ref_mbea <file.adj> 2 <uvtrans> <order> <stride> <first> <count> <threads> <max_root>
#include <omp.h>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

// The per-root entry point and the counter are private/protected members of
// the reference's classes; this driver calls them directly.
#define private public
#define protected public
#include "BiGraph.h"
#include "BicliqueFinder.h"
#undef private
#undef protected

static int run_samples(CSRBiGraph* graph, int stride, const std::vector<int>& offsets,
                       int threads, double max_root_arg) {
  if (stride < 1 || offsets.empty() || threads < 1) return 2;
  long long max_root = max_root_arg > 0 && max_root_arg < 1
                           ? (long long)(max_root_arg * graph->V_size)
                           : (long long)max_root_arg;
  if (max_root <= 0 || max_root > graph->V_size) max_root = graph->V_size;
  std::vector<MbeaFinderBitset*> finders;
  for (int t = 0; t < threads; ++t) finders.push_back(new MbeaFinderBitset(graph));
  for (int j : offsets) {
    if (j < 0) return 2;
    std::vector<int> roots;
    for (long long v = j % stride; v < max_root; v += stride) roots.push_back((int)v);
    for (auto* f : finders) f->maximal_nodes_ = 0;
    const double t0 = get_cur_time();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
    for (int k = 0; k < (int)roots.size(); ++k) {
      const int v = roots[k];
      MbeaFinderBitset* f = finders[omp_get_thread_num()];
      std::vector<int> L(graph->column_indices + graph->row_offset[v],
                         graph->column_indices + graph->row_offset[v + 1]);
      if (!L.empty()) f->biclique_find(L, v, 0);
    }
    const double dt = get_cur_time() - t0;
    long long cnt = 0;
    for (auto* f : finders) cnt += f->maximal_nodes_;
    printf("sample %d roots %zu count %lld seconds %.6f\n", j, roots.size(), cnt, dt);
    fflush(stdout);
  }
  for (auto* f : finders) delete f;
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s <file.adj> <sel 0|1> [uvtrans] [order]\n", argv[0]);
    return 2;
  }
  const int sel = atoi(argv[2]);
  if (sel == 2 && argc != 10) {
    fprintf(stderr, "usage: %s <file.adj> 2 <uvtrans> <order> <stride> <first> <count> "
                    "<threads> <max_root>\n", argv[0]);
    return 2;
  }
  Option opt;
  opt.fast_mode = 1;
  opt.uvtrans = argc > 3 ? atoi(argv[3]) : 0;
  opt.order = argc > 4 ? atoi(argv[4]) : 1;
  CSRBiGraph* graph = new CSRBiGraph();
  const double t0 = get_cur_time();
  graph->Read(argv[1], opt);
  int rc = 0;
  if (sel == 2) {
    printf("read seconds %.3f V %d U %d E %d\n", get_cur_time() - t0, graph->V_size,
           graph->U_size, graph->edge_size);
    fflush(stdout);
    std::vector<int> offsets;
    const std::string first = argv[6];
    if (first.find(',') != std::string::npos) {
      std::stringstream ss(first);
      std::string item;
      while (std::getline(ss, item, ',')) offsets.push_back(atoi(item.c_str()));
    } else {
      for (int j = atoi(argv[6]); j < atoi(argv[6]) + atoi(argv[7]); ++j) offsets.push_back(j);
    }
    rc = run_samples(graph, atoi(argv[5]), offsets, atoi(argv[8]), atof(argv[9]));
  } else {
    BicliqueFinder* finder = nullptr;
    if (sel == 0)
      finder = new MbeaFinder(graph);
    else
      finder = new MbeaFinderBitset(graph);
    finder->Execute();
    finder->PrintResult();
    delete finder;
  }
  graph->Reset();
  delete graph;
  return rc;
}
