// xtric: the single-GPU command-line driver. Same flags, messages and output
// lines as the reference's main.cpp (main.cpp:49-276), one process:
//   xtric -f graph.bin [-b|-d] [-r n] [-s bufsize]
//   xtric -n N [-l] [-p pct]
// -b/-d/-r/-s shape the reference's multi-rank partitioning and buffers and
// are accepted and ignored with a notice. The -f file is streamed to the
// device and parsed there, and the -n graph (without -p random edges) is
// generated on the device. Extra long options:
//   --orient id|degree   orientation of the device CSR (default degree)
//   --nprocs P           strip ranks the -n graph is generated for (default 1)
//   --radius R           RGG radius instead of the reference's r(n)
//   --seed S             seed of the -p random edges (default 1)
//   --int32              read a USE_32_BIT_GRAPH vite file
//   --per-vertex FILE    write per-vertex counts, one per line
#include <getopt.h>
#include <unistd.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <memory>
#include <string>

#include "xtric_host.hpp"

using namespace xtb200;

namespace {

std::string inputFileName, perVertexFile;
GraphElem nvRGG = 0;
bool generateGraph = false, readBalanced = false, readBalancedDynamic = false, randomNumberLCG = false;
GraphWeight randomEdgePercent = 0.0;
long bufferSize = -1;
int ranksPerNode = 1, nprocsRGG = 1, orient = XT_ORIENT_DEGREE, elemBytes = 8;
double radius = 0.0;
uint64_t seed = 1;

[[noreturn]] void abort_run() {
  std::cout.flush();
  std::exit(157);  // the exit status MPI_Abort(comm, -99) gives one process
}

double now() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

void parseCommandLine(int argc, char *const argv[]) {
  static option longopts[] = {{"orient", required_argument, nullptr, 1000},
                              {"nprocs", required_argument, nullptr, 1001},
                              {"radius", required_argument, nullptr, 1002},
                              {"seed", required_argument, nullptr, 1003},
                              {"int32", no_argument, nullptr, 1004},
                              {"per-vertex", required_argument, nullptr, 1005},
                              {nullptr, 0, nullptr, 0}};
  int ret;
  while ((ret = getopt_long(argc, argv, "f:r:n:p:olbds:", longopts, nullptr)) != -1) {
    switch (ret) {
      case 'f': inputFileName.assign(optarg); break;
      case 'b': readBalanced = true; break;
      case 'd': readBalancedDynamic = true; break;
      case 'r': ranksPerNode = atoi(optarg); break;
      case 'n':
        nvRGG = atol(optarg);
        if (nvRGG > 0) generateGraph = true;
        break;
      case 'l': randomNumberLCG = true; break;
      case 'p': randomEdgePercent = atof(optarg); break;
      case 's': bufferSize = atol(optarg); break;
      case 'o': break;
      case 1000: orient = std::string(optarg) == "id" ? XT_ORIENT_ID : XT_ORIENT_DEGREE; break;
      case 1001: nprocsRGG = atoi(optarg); break;
      case 1002: radius = atof(optarg); break;
      case 1003: seed = strtoull(optarg, nullptr, 10); break;
      case 1004: elemBytes = 4; break;
      case 1005: perVertexFile.assign(optarg); break;
      default:
        std::cerr << "Unknown option." << std::endl;
        abort_run();
    }
  }
  if (generateGraph && (readBalanced || readBalancedDynamic))
    std::cout << "Balanced read (option -b) is only applicable for real-world graphs. "
              << "This option does nothing for generated (synthetic) graphs." << std::endl;
  if (argc == 1) {
    std::cerr << "Must specify some options." << std::endl;
    abort_run();
  }
  if (!generateGraph && inputFileName.empty()) {
    std::cerr << "Must specify a binary file name with -f or provide parameters for generating a graph." << std::endl;
    abort_run();
  }
  if (!generateGraph && randomNumberLCG) {
    std::cerr << "Must specify -g for graph generation using LCG." << std::endl;
    abort_run();
  }
  if (!generateGraph && (randomEdgePercent > 0.0)) {
    std::cerr << "Must specify -g for graph generation first to add random edges to it." << std::endl;
    abort_run();
  }
  if (generateGraph && ((randomEdgePercent < 0.0) || (randomEdgePercent >= 100.0))) {
    std::cerr << "Invalid random edge percentage for generated graph!" << std::endl;
    abort_run();
  }
  if (bufferSize != -1 || ranksPerNode != 1 || readBalanced || readBalancedDynamic)
    std::cout << "*Warning*: -b/-d/-r/-s configure multi-rank runs and are ignored on one GPU." << std::endl;
}

}  // namespace

int main(int argc, char *argv[]) {
  parseCommandLine(argc, argv);
  // -f and -n without random edges are read or generated on the device (the
  // host never holds the graph); -n with -p > 0 generates on the host, as
  // its random edges come from a host RNG
  const bool on_device = !generateGraph || randomEdgePercent <= 0.0;
  if (generateGraph && (nprocsRGG <= 0 || (nprocsRGG & (nprocsRGG - 1)))) {
    std::cout << "Error: random geometric graph generation require power-of-2 #processes." << std::endl;
    abort_run();
  }
  if (generateGraph && !randomNumberLCG)
    std::cerr << "*Warning*: coordinates are always drawn from the reference's LCG (-l); the reference's "
                 "std::random_device path is not reproducible."
              << std::endl;
  Graph *g = nullptr;
  std::unique_ptr<TriangleCountingSingle> tr;
  GraphElem nv = 0, ne = 0;
  const double td0 = now();
  try {
    if (on_device) {
      if (generateGraph) tr.reset(new TriangleCountingSingle(nvRGG, nprocsRGG, radius, orient));
      else tr.reset(new TriangleCountingSingle(inputFileName, elemBytes, orient));
      const xt_graph_info inf = tr->info();
      nv = inf.nv;
      ne = inf.n_input;
    } else {
      GenerateRGG gr(nvRGG, nprocsRGG, radius, seed);
      g = gr.generate(true, true, randomEdgePercent);
      nv = g->get_nv();
      ne = g->get_ne();
    }
  } catch (const Error &e) {
    if (!generateGraph) std::cout << " Error opening file! " << std::endl;
    std::cerr << e.what() << std::endl;
    abort_run();
  }
  Graph::print_dist_stats(nv, ne);
  const double tdt = now() - td0;
  if (!generateGraph)
    std::cout << "Time to read input file and create distributed graph (secs.): " << tdt << std::endl;
  else
    std::cout << "Time to generate distributed graph of " << nvRGG << " vertices (secs.): " << tdt << std::endl;

  try {
    if (!tr) tr.reset(new TriangleCountingSingle(g, orient));
    std::vector<GraphElem> pv;
    const double t0 = now();
    const GraphElem ntris = perVertexFile.empty() ? tr->count() : tr->count(pv);
    const double t = now() - t0;
    std::cout << "Avg/Min/Max execution time (secs.) for triangle counting on 1 processes: " << t << ", " << t
              << ", " << t << std::endl;
    std::cout << "Number of triangles: " << ntris << std::endl;
    std::cout << "TEPS: " << double(ne) / t << std::endl;
    if (!perVertexFile.empty()) {
      std::ofstream f(perVertexFile);
      for (GraphElem c : pv) f << c << "\n";
    }
    tr->clear();
  } catch (const Error &e) {
    std::cerr << e.what() << std::endl;
    delete g;
    return 2;
  }
  delete g;
  return 0;
}
