// Header-only C++ mirror of the reference's single-device API surface on top
// of the C ABI in include/xtric.h:
//   Graph                  - the CSR interface of graph.hpp:52-275
//   BinaryEdgeList::read   - the vite reader of graph.hpp:294-395
//   GenerateRGG::generate  - the RGG generator of graph.hpp:745-1364
//   TriangleCountingSingle - the engine of xxtric-gpu.hpp:22-298
// so a main.cpp-style driver swaps its includes and keeps its code.
#pragma once

#include <cmath>
#include <cstdint>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/xtric.h"

namespace xtb200 {

using GraphElem = int64_t;
using GraphWeight = double;

struct Edge {
  GraphElem tail_;
  GraphWeight weight_;
};

class Error : public std::runtime_error {
 public:
  Error(xt_status s, const std::string &what) : std::runtime_error(what), status(s) {}
  xt_status status;
};

inline void check(xt_status s, const std::string &what, const xt_ctx *ctx = nullptr) {
  if (s != XT_OK) {
    std::string msg = what + ": " + xt_strerror(s);
    if (ctx && xt_last_error(ctx)[0]) msg += std::string(" (") + xt_last_error(ctx) + ")";
    throw Error(s, msg);
  }
}

// One process owns every vertex, so local and global ids coincide.
class Graph {
 public:
  Graph(GraphElem nv, GraphElem ne) : nv_(nv), ne_(ne), edge_indices_(size_t(nv + 1), 0), tails_(size_t(ne)) {}

  void edge_range(GraphElem v, GraphElem &e0, GraphElem &e1) const {
    e0 = edge_indices_[size_t(v)];
    e1 = edge_indices_[size_t(v) + 1];
  }
  Edge get_edge(GraphElem i) const { return Edge{tails_[size_t(i)], 1.0}; }
  GraphElem get_nv() const { return nv_; }
  GraphElem get_ne() const { return ne_; }
  GraphElem get_lnv() const { return nv_; }
  GraphElem get_lne() const { return ne_; }
  GraphElem local_to_global(GraphElem i) const { return i; }
  GraphElem global_to_local(GraphElem i) const { return i; }
  int get_owner(GraphElem) const { return 0; }

  // the statistics block of graph.hpp:230-264 for one process
  void print_dist_stats() const { print_dist_stats(nv_, ne_); }
  static void print_dist_stats(GraphElem nv_, GraphElem ne_) {
    const double average = double(ne_), avg_sq = double(ne_) * double(ne_);
    const double var = std::fabs(avg_sq - average * average), stddev = std::sqrt(var);
    std::cout << "\n-------------------------------------------------------\n"
              << "Graph edge distribution characteristics\n"
              << "-------------------------------------------------------\n"
              << "Number of vertices: " << nv_ << "\n"
              << "Number of edges: " << ne_ << "\n"
              << "Maximum number of edges: " << ne_ << "\n"
              << "Average number of edges: " << average << "\n"
              << "Expected value of X^2: " << avg_sq << "\n"
              << "Variance: " << var << "\n"
              << "Standard deviation: " << stddev << "\n"
              << "-------------------------------------------------------" << std::endl;
  }

  GraphElem nv_, ne_;
  std::vector<GraphElem> edge_indices_;
  std::vector<GraphElem> tails_;
};

class BinaryEdgeList {
 public:
  explicit BinaryEdgeList(int elem_bytes = 8) : elem_bytes_(elem_bytes) {}
  // me/nprocs/ranks_per_node are accepted for signature parity; one process
  // reads the whole file
  Graph *read(int /*me*/, int /*nprocs*/, int /*ranks_per_node*/, const std::string &file) {
    int64_t nv = 0, ne = 0;
    check(xt_vite_read(file.c_str(), elem_bytes_, &nv, &ne, nullptr, nullptr), "reading " + file);
    Graph *g = new Graph(nv, ne);
    check(xt_vite_read(file.c_str(), elem_bytes_, &nv, &ne, g->edge_indices_.data(), g->tails_.data()),
          "reading " + file);
    return g;
  }

 private:
  int elem_bytes_;
};

class GenerateRGG {
 public:
  // nprocs: the strip-rank count the graph is generated for (the reference's
  // graph depends on mpiexec -n); radius <= 0: the reference's r(n)
  explicit GenerateRGG(GraphElem nv, int nprocs = 1, double radius = 0.0, uint64_t seed = 1)
      : nv_(nv), nprocs_(nprocs), radius_(radius), seed_(seed) {}

  Graph *generate(bool isLCG, bool /*unitEdgeWeight*/ = true, GraphWeight randomEdgePercent = 0.0) {
    if (!isLCG)
      std::cerr << "*Warning*: coordinates are always drawn from the reference's LCG (-l); the reference's "
                   "std::random_device path is not reproducible."
                << std::endl;
    int64_t ne = 0;
    check(xt_rgg_generate(nv_, nprocs_, radius_, randomEdgePercent, seed_, 0, &ne, nullptr, nullptr),
          "generating the random geometric graph");
    Graph *g = new Graph(nv_, ne);
    check(xt_rgg_generate(nv_, nprocs_, radius_, randomEdgePercent, seed_, ne, &ne, g->edge_indices_.data(),
                          g->tails_.data()),
          "generating the random geometric graph");
    return g;
  }

 private:
  GraphElem nv_;
  int nprocs_;
  double radius_;
  uint64_t seed_;
};

// TriangleCountingSingle: the constructor builds the oriented device CSR
// (canonicalising the input: the reference trusts it), count() runs the
// device count, clear() releases the device memory.
class TriangleCountingSingle {
 public:
  explicit TriangleCountingSingle(Graph *g, int orient = XT_ORIENT_DEGREE, int device = 0) {
    check(xt_open(device, &ctx_), "opening the CUDA device");
    built(xt_graph_from_csr(ctx_, g->get_nv(), g->edge_indices_.data(), g->tails_.data(), 0, orient, &dg_));
  }
  // A vite file (BinaryEdgeList's format, elem_bytes 8 or 4) streamed to the
  // device and parsed there: the host holds no copy of the graph.
  TriangleCountingSingle(const std::string &vite_path, int elem_bytes, int orient = XT_ORIENT_DEGREE,
                         int device = 0) {
    check(xt_open(device, &ctx_), "opening the CUDA device");
    built(xt_graph_from_vite(ctx_, vite_path.c_str(), elem_bytes, 0, orient, &dg_));
  }
  // The reference's random geometric graph (no random edges) generated and
  // built on the device, as nprocs strip ranks make it.
  TriangleCountingSingle(GraphElem nv, int nprocs, double radius, int orient = XT_ORIENT_DEGREE, int device = 0) {
    check(xt_open(device, &ctx_), "opening the CUDA device");
    built(xt_graph_from_rgg(ctx_, nv, nprocs, radius, orient, &dg_));
  }
  ~TriangleCountingSingle() { clear(); }
  TriangleCountingSingle(const TriangleCountingSingle &) = delete;
  TriangleCountingSingle &operator=(const TriangleCountingSingle &) = delete;

  GraphElem count() {
    int64_t t = 0;
    check(xt_count(dg_, &t, nullptr), "counting", ctx_);
    return t;
  }
  // per-vertex counts (each triangle credits its three corners)
  GraphElem count(std::vector<GraphElem> &per_vertex) {
    per_vertex.assign(size_t(info().nv), 0);
    int64_t t = 0;
    check(xt_count(dg_, &t, per_vertex.data()), "counting", ctx_);
    return t;
  }
  // triangles on every oriented edge (k-truss support), in the order of the
  // library's oriented CSR (internal numbering, see xt_graph_get_csr/_perm)
  GraphElem count_edges(std::vector<GraphElem> &support) {
    support.assign(size_t(info().n_edges), 0);
    int64_t t = 0;
    check(xt_count_edges(dg_, &t, support.data()), "counting", ctx_);
    return t;
  }
  xt_graph_info info() const {
    xt_graph_info i{};
    xt_graph_get_info(dg_, &i);
    return i;
  }
  void clear() {
    if (dg_) xt_graph_free(dg_);
    dg_ = nullptr;
    if (ctx_) xt_close(ctx_);
    ctx_ = nullptr;
  }

 private:
  void built(xt_status s) {
    if (s != XT_OK) {
      std::string msg = std::string("building the device graph: ") + xt_strerror(s) + " (" + xt_last_error(ctx_) + ")";
      xt_close(ctx_);
      ctx_ = nullptr;
      throw Error(s, msg);
    }
  }
  xt_ctx *ctx_ = nullptr;
  xt_graph *dg_ = nullptr;
};

// Many graphs counted in one launch: graph g has vertices
// [vertex_offsets[g], vertex_offsets[g+1]) and rows [edge_offsets[g],
// edge_offsets[g+1]) of src/dst (graph-local ids). Returns the total and
// fills per_graph.
inline GraphElem BatchCount(const std::vector<int64_t> &vertex_offsets, const std::vector<int64_t> &edge_offsets,
                            const std::vector<int32_t> &src, const std::vector<int32_t> &dst,
                            std::vector<GraphElem> &per_graph, int orient = XT_ORIENT_DEGREE, int device = 0) {
  xt_ctx *ctx = nullptr;
  check(xt_open(device, &ctx), "opening the CUDA device");
  const int64_t ng = int64_t(vertex_offsets.size()) - 1;
  per_graph.assign(size_t(ng > 0 ? ng : 0), 0);
  int64_t t = 0;
  const xt_status s = xt_batch_count(ctx, ng, vertex_offsets.data(), edge_offsets.data(), src.data(), dst.data(),
                                     orient, &t, per_graph.data());
  const std::string detail = xt_last_error(ctx);
  xt_close(ctx);
  if (s != XT_OK) throw Error(s, std::string("batch count: ") + xt_strerror(s) + " (" + detail + ")");
  return t;
}

// Count queries served by device-memory-budget admission and continuous
// batching (xt_serve_*): submit() returns a ticket, wait() its count. The
// query's edge rows are read while it runs: keep them alive until wait().
class Server {
 public:
  explicit Server(int device = 0, int64_t budget_bytes = 0, int slots = 0, int orient = XT_ORIENT_DEGREE) {
    xt_serve_config c{};
    c.budget_bytes = budget_bytes;
    c.slots = slots;
    c.orient = orient;
    check(xt_serve_open(device, &c, &srv_), "opening the server");
  }
  ~Server() {
    if (srv_) xt_serve_close(srv_);
  }
  Server(const Server &) = delete;
  Server &operator=(const Server &) = delete;
  int64_t submit(int64_t nv, const std::vector<int32_t> &src, const std::vector<int32_t> &dst) {
    if (src.size() != dst.size()) throw Error(XT_ERR_INVALID, "src and dst differ in length");
    int64_t ticket = 0;
    check(xt_serve_submit(srv_, nv, int64_t(src.size()), src.data(), dst.data(), &ticket), "submitting");
    return ticket;
  }
  // the count of the query (blocks); latency_s receives submit-to-result seconds
  GraphElem wait(int64_t ticket, double *latency_s = nullptr) {
    int64_t c = 0;
    double lat = 0;
    check(xt_serve_wait(srv_, ticket, -1, &c, &lat), "query");
    if (latency_s) *latency_s = lat;
    return c;
  }
  xt_serve_stats stats() {
    xt_serve_stats s{};
    check(xt_serve_get_stats(srv_, &s), "server statistics");
    return s;
  }

 private:
  xt_server *srv_ = nullptr;
};

}  // namespace xtb200
