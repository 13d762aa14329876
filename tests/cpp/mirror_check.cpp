// Exercises the C++ host mirror (xxtric_b200/host/xtric_host.hpp) beyond the
// reference's TriangleCountingSingle: the per-edge count, the one-call batch
// count and the query server. Prints one line per result; on a library error
// prints "error <status>" and exits 3 (no device: status 9).
#include <cstdio>

#include "xxtric_b200/host/xtric_host.hpp"

int main() {
  using namespace xtb200;
  try {
    // two graphs as one batch: K4 (4 triangles) and a triangle
    const std::vector<int64_t> voff{0, 4, 7}, eoff{0, 6, 9};
    const std::vector<int32_t> src{0, 0, 0, 1, 1, 2, 0, 1, 2}, dst{1, 2, 3, 2, 3, 3, 1, 2, 0};
    std::vector<GraphElem> per;
    const GraphElem t = BatchCount(voff, eoff, src, dst, per);
    std::printf("batch %lld %lld %lld\n", (long long)t, (long long)per[0], (long long)per[1]);
    // K4 as the reference's CSR: every edge is in 2 triangles
    Graph g(4, 12);
    const GraphElem rows[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
    for (int v = 0; v < 4; v++) {
      g.edge_indices_[v + 1] = 3 * (v + 1);
      for (int k = 0; k < 3; k++) g.tails_[3 * v + k] = rows[v][k];
    }
    TriangleCountingSingle tc(&g);
    std::vector<GraphElem> sup;
    const GraphElem te = tc.count_edges(sup);
    long long ssum = 0;
    for (GraphElem x : sup) ssum += x;
    std::printf("edges %lld %zu %lld\n", (long long)te, sup.size(), ssum);
    Server srv;
    const std::vector<int32_t> s1{0, 0, 0, 1, 1, 2}, d1{1, 2, 3, 2, 3, 3};
    const int64_t tk = srv.submit(4, s1, d1);
    double lat = 0;
    const GraphElem served = srv.wait(tk, &lat);
    std::printf("served %lld %d\n", (long long)served, lat > 0 ? 1 : 0);
  } catch (const Error &e) {
    std::printf("error %d %s\n", int(e.status), e.what());
    return 3;
  }
  return 0;
}
