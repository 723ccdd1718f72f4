// Host-only driver for the reference's in-tree CPU enumerators.
//
// TEST INFRASTRUCTURE ONLY: built by oracle/Makefile (target `ref`) against
// the reference's own sources (src/BiGraph.cu, src/BicliqueFinder.cu,
// src/Utility.cu), output into oracle/_ref/.  It reads an .adj file with
// CSRBiGraph::Read (fast mode) and runs MbeaFinder (sel 0, src/BicliqueFinder.cu:20-57)
// or MbeaFinderBitset (sel 1, src/BicliqueFinder.cu:59-197), printing the
// reference's own result lines ("Total processing time", "maximal nodes").
//
// usage: ref_mbea <file.adj> <sel 0|1> [uvtrans] [order]
#include <cstdio>
#include <cstdlib>

#include "BiGraph.h"
#include "BicliqueFinder.h"

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s <file.adj> <sel 0|1> [uvtrans] [order]\n", argv[0]);
    return 2;
  }
  Option opt;
  opt.fast_mode = 1;
  opt.uvtrans = argc > 3 ? atoi(argv[3]) : 0;
  opt.order = argc > 4 ? atoi(argv[4]) : 1;
  CSRBiGraph* graph = new CSRBiGraph();
  graph->Read(argv[1], opt);
  BicliqueFinder* finder = nullptr;
  if (atoi(argv[2]) == 0)
    finder = new MbeaFinder(graph);
  else
    finder = new MbeaFinderBitset(graph);
  finder->Execute();
  finder->PrintResult();
  delete finder;
  graph->Reset();
  delete graph;
  return 0;
}
