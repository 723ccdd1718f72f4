// MBE_GPU: drop-in command line of the reference (src/main.cu:76-149).
//
//   MBE_GPU -i <file.adj> [-s 0|1|2|3] [-t 0|1|2] [-o 0|1|2|3] [-f] [-p]
//           [-m bound_height] [-n bound_size] [-x ngpus]
//
// Flags, defaults and output lines follow the reference; -m and -n are
// parsed here (the reference's getopt string omits them, src/main.cu:95).
// All selectors run the one persistent engine: -s 2 with the given bounds,
// -s 0 and -s 1 without task splitting, -s 3 (multi-GPU) on one GPU.
#include <signal.h>
#include <sys/time.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "mbe_finder.h"

namespace {
double wall_s() {
  struct timeval tv;
  gettimeofday(&tv, nullptr);
  return (double)tv.tv_sec + (double)tv.tv_usec * 1e-6;
}
void on_sigterm(int) {
  printf("Total processing time is more than 7200s\n");
  exit(0);
}
}  // namespace

int main(int argc, char* argv[]) {
  signal(SIGTERM, on_sigterm);
  int ngpus = 1, op, sel = 0, bound_height = 20, bound_size = 1500;
  bool print_sm_time = false;
  Option opt;
  char graph_name[4096] = "db/Writers.adj";
  while ((op = getopt(argc, argv, "h:x:i:s:t:o:fpm:n:")) != -1) {
    switch (op) {
      case 'i':
        snprintf(graph_name, sizeof(graph_name), "%s", optarg);
        break;
      case 't':
        opt.uvtrans = atoi(optarg);
        break;
      case 's':
        sel = atoi(optarg);
        break;
      case 'o':
        opt.order = atoi(optarg);
        break;
      case 'f':
        opt.fast_mode = 1;
        break;
      case 'm':
        bound_height = atoi(optarg);
        break;
      case 'n':
        bound_size = atoi(optarg);
        break;
      case 'x':
        ngpus = atoi(optarg);
        break;
      case 'p':
        print_sm_time = true;
        break;
      default:
        break;
    }
  }
  double start_t = wall_s();
  CSRBiGraph* graph = new CSRBiGraph();
  int rc = graph->Read(graph_name, opt);
  printf("Max blocks:%u Warps per block:%u Max1d:0x%x Max2d:0x%x\n", 0u, 16u,
         (unsigned)graph->V_degree, (unsigned)graph->U_degree);
  printf("trans:%d sel:%d order:%d fast_mode:%d\n", opt.uvtrans, sel, opt.order, opt.fast_mode);
  printf("Graph load time: %lf s\n", wall_s() - start_t);
  if (rc != MBE_OK) {
    delete graph;
    return 1;
  }
  if (sel == 3 && ngpus > 1) printf("multi-GPU mode runs on one GPU in this build\n");
  IterFinderGpu6* finder = (sel == 0 || sel == 1) ? new IterFinderGpu(graph)
                                                   : new IterFinderGpu6(graph, bound_height, bound_size);
  finder->params().sm_timing = print_sm_time ? 1 : 0;
  printf("large worklist size: %d local tiny size: %d\n", 0, 0);
  finder->Execute();
  if (finder->status() != MBE_OK) {
    fprintf(stderr, "enumeration failed: %s\n", finder->last_error().c_str());
    delete finder;
    delete graph;
    return 1;
  }
  const mbe_result& r = finder->result();
  if (print_sm_time) {
    printf("SM exit: %lf\n", r.sm_exit_min_ms);
    printf("SM exit: %lf\n", r.sm_exit_max_ms);
  }
  printf("%d\n", 0);
  printf("non_maximal: %llu\n", (unsigned long long)r.non_maximal);
  printf("set hash: 0x%016llx\n", (unsigned long long)r.set_hash);
  finder->PrintResult();
  delete finder;
  delete graph;
  return 0;
}
