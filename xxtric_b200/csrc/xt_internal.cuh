// Internal declarations shared by the translation units of libxtb200.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>
#include <unordered_map>

#include "../../include/xtric.h"

namespace xt {

constexpr int kWarp = 32;
// int32 column arrays carry this many spare entries past their end
constexpr size_t kColPad = 8;

// ---- context ---------------------------------------------------------------
struct Ctx {
  int device = 0;
  int sm_count = 148;
  size_t smem_optin = 0;  // max dynamic shared memory per block (opt-in)
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaStream_t copy_stream = nullptr;  // host-to-device copies that overlap the build (created on first use)
  std::string last_error;
  int64_t fail_alloc_countdown = 0;  // test hook: >0 counts down to a failing allocation
  // device-side error word reused by kernels that check their own inputs
  int *d_err = nullptr;
  int64_t launches = 0;  // kernels of this library launched on this context
  // device bytes this context holds (its own allocations) and their high-water mark
  std::unordered_map<void *, size_t> live;
  int64_t bytes_live = 0, bytes_peak = 0;
  // optional totals shared by several contexts (a server's slots): bytes live
  // in all of them together and the high-water mark of that sum
  std::atomic<int64_t> *shared_live = nullptr, *shared_peak = nullptr;
};

// Launch-configuration wrapper that counts the library's own kernel launches.
inline dim3 counted(Ctx *c, dim3 grid) {
  c->launches++;
  return grid;
}

// Stream-ordered device allocation with the context's failure hook.
xt_status dalloc(Ctx *c, void **p, size_t bytes);
void dfree(Ctx *c, void *p);

template <class T>
xt_status dalloc_n(Ctx *c, T **p, size_t n) {
  return dalloc(c, reinterpret_cast<void **>(p), n * sizeof(T));
}

// Records a CUDA error (if any) and converts it to a status.
xt_status cuda_status(Ctx *c, cudaError_t e, const char *what);
xt_status set_error(Ctx *c, xt_status s, const std::string &msg);

#define XT_CUDA(ctx, call)                                   \
  do {                                                       \
    cudaError_t xt_e_ = (call);                              \
    if (xt_e_ != cudaSuccess) return xt::cuda_status((ctx), xt_e_, #call); \
  } while (0)

#define XT_TRY(expr)                  \
  do {                                \
    xt_status xt_s_ = (expr);         \
    if (xt_s_ != XT_OK) return xt_s_; \
  } while (0)

// ---- oriented graph on the device ------------------------------------------
struct Plan;  // degree-binned schedule, built once per graph

// Pad value of the padded column array: negative, so below every vertex id
// (no membership test accepts it).
constexpr int32_t kPadSentinel = -2;

// In-record of edge u->v, stored with the head v: the columns of N+(u) that
// rank above v, i.e. the suffix d_colp[s, s+len) after v's own position
// (s indexes the padded column array).
// Every triangle (u,v,w) has its w in exactly this suffix and in N+(v).
// Packed in 8 bytes: pair = s / 8 (the 32-byte pair the suffix starts in)
// and lw = len | (s % 8) << kRecLenBits, so s < 2^35 and len < 2^29. The
// tail u is kept apart (Graph::d_irec_u), built when a per-vertex or
// per-edge count first needs it.
struct __align__(8) InRec {
  uint32_t pair;
  uint32_t lw;
};
constexpr int kRecLenBits = 29;
constexpr int64_t kMaxColp = int64_t(1) << 35;      // padded columns the records can address
constexpr int64_t kMaxRecLen = int64_t(1) << kRecLenBits;
__host__ __device__ inline InRec make_inrec(int64_t s, int64_t len) {
  InRec r;
  r.pair = uint32_t(s >> 3);
  r.lw = uint32_t(len) | (uint32_t(s & 7) << kRecLenBits);
  return r;
}
__host__ __device__ inline int64_t rec_s(InRec r) { return (int64_t(r.pair) << 3) | int64_t(r.lw >> kRecLenBits); }
__host__ __device__ inline int32_t rec_len(InRec r) { return int32_t(r.lw & uint32_t(kMaxRecLen - 1)); }

struct Graph {
  Ctx *ctx = nullptr;
  int64_t nv = 0;
  int64_t n_input = 0;
  int64_t ne = 0;  // |E+|
  int orient = XT_ORIENT_DEGREE;
  // Vertices are renumbered so that the orientation rank IS the id: under
  // XT_ORIENT_DEGREE, internal id = position in (degree, input id) order;
  // under XT_ORIENT_ID the numbering is the input's. Every edge then points
  // from the lower to the higher internal id and rows ascend by rank.
  int64_t *d_off = nullptr;   // out-CSR offsets, nv+1
  int32_t *d_col = nullptr;   // out-CSR columns N+(u), ne (+kColPad), rows ascending
  int64_t *d_ioff = nullptr;  // in-record offsets per head v, nv+1
  InRec *d_irec = nullptr;    // one record per edge u->v, grouped by v (ne + 2: the last 16 bytes are slack
                              //   for 16-byte aligned bulk prefetches)
  int32_t *d_irec_u = nullptr;  // the tail u of each record, built on first use (per-vertex, per-edge)
  // The columns again, each row starting on an 8-column (32-byte) boundary
  // and padded with kPadSentinel: the count streams suffixes from here in
  // whole 32-byte pairs without masking. d_poff[u] is row u's start.
  int32_t *d_colp = nullptr;
  int64_t *d_poff = nullptr;  // nv+1
  int32_t *d_perm = nullptr;  // internal id -> input id (null when identity)
  int64_t max_degree = 0;
  int64_t max_out_degree = 0;
  int64_t max_in_degree = 0;
  int64_t tune_block_work = 0;  // schedule overrides (0: choose automatically)
  int64_t tune_warp_work = 0;
  int64_t tune_bitmap_bits = 0;
  int prefetch_suffix = 0;      // global count: bulk L2 prefetch of each record's suffix (1) or not (0)
  int lane_merge = 0;            // lane tasks: two-pointer merge (1) or binary search (0) over N+(v)
  int cluster_tier = 0;         // global count: heads over a CTA's member set on thread-block clusters (1) or
                                //   as CTA tasks over parts of their members (0, the default: faster)
  int cuckoo_iters = -1;        // test hook: cuckoo eviction chain limit (-1: the default)
  int claim_block = 0;          // warp tasks taken per atomic on their cursor (0: 4 for a batch, else 1)
  int64_t tier_lane_work = -1;  // tier limits (-1: automatic, 0: tier off)
  int64_t tier_warp_work = -1;
  int32_t *d_group = nullptr;   // internal id -> group (graph of a batch), or null
  int64_t n_groups = 0;
  // a captured count (CUDA graph) writing the total and the per-group
  // counts into d_res[0] and d_res[1..n_groups]
  cudaGraphExec_t exec = nullptr;
  int64_t exec_kernels = 0;  // library kernels inside `exec`, counted per replay
  int64_t *d_res = nullptr;
  int64_t wedge_work = 0;   // sum over oriented (u,v) of d+(v)
  int64_t stream_work = 0;  // sum over u of C(d+(u), 2): the suffix columns the count streams
  int64_t colp_len = 0;     // entries of the padded column array
  Plan *plan = nullptr;
};

// Optional: the rows still in host memory. build_from_edges then copies
// them into d_src/d_dst (device buffers of ne rows) in chunks on the
// context's copy stream and turns each chunk into keys as soon as it lands,
// so key generation overlaps the copy-in.
struct HostRows {
  const int32_t *src, *dst;
};

// Builds the oriented CSR from a device edge list (int32 ids) of ne rows.
// Rows may repeat, be one-directional or self loops.
xt_status build_from_edges(Ctx *c, int64_t nv, int64_t ne, const int32_t *d_src, const int32_t *d_dst,
                           int orient, Graph *g, const HostRows *upload = nullptr);
// Builds from a device CSR (int64 offsets and tails). canonical: rows already
// sorted, deduped, symmetric and loop-free, so no sort is needed.
xt_status build_from_csr(Ctx *c, int64_t nv, const int64_t *d_off, const int64_t *d_tails, bool canonical,
                         int orient, Graph *g);
void free_graph_device(Graph *g);
// Reads a vite binary file (8- or 4-byte fields) through pinned staging
// buffers into a device CSR and builds from it (vite.cu).
xt_status build_from_vite(Ctx *c, const char *path, int elem_bytes, bool canonical, int orient, Graph *g);

// Builds the disjoint union of ng graphs (host offset tables, device edge
// rows with graph-local ids) as one graph with a per-vertex group map.
xt_status build_batch(Ctx *c, int64_t ng, const int64_t *h_voff, const int64_t *h_eoff, const int32_t *d_src,
                      const int32_t *d_dst, int orient, Graph *g);

// Builds (or rebuilds) the per-graph schedule and graph statistics.
xt_status make_plan(Graph *g);
void free_plan(Graph *g);

// Launches the count on the graph's context stream. d_global: one int64
// (overwritten); d_pv: nv int64 (nullable, overwritten).
// d_groups: n_groups int64 per-group counts (graphs built as a batch), nullable.
// d_support: ne int64, the triangles on each oriented edge in out-CSR order
// (nullable; not together with d_pv).
// shard / nshards: count only every nshards-th task of the schedule from
// task `shard` on (each tier's list alike); the nshards shards' outputs sum
// to the whole count's.
xt_status count_graph(Graph *g, int64_t *d_global, int64_t *d_pv, int64_t *d_groups = nullptr,
                      int64_t *d_support = nullptr, int shard = 0, int nshards = 1);
// Synchronises the context stream and reports a count whose bounded device
// wait gave up (XT_ERR_TIMEOUT); the synchronous count calls end with it.
xt_status count_status(Ctx *c);
// tasks of the global count's thread-block cluster tier in the graph's plan (0 without a plan)
int64_t cluster_task_count(const Graph *g);
// lane tasks in the graph's plan (0 without a plan)
int64_t lane_task_count(const Graph *g);

}  // namespace xt

// The host set-up of the reference's random geometric graph (host_io.cpp):
// radius, each strip rank's first LCG value and its strip [lo, lo + range).
xt_status xt_rgg_setup(int64_t nv, int nprocs, double radius, double *rn, int64_t *x0, double *lo, double *range);

struct xt_ctx {
  xt::Ctx c;
};
struct xt_graph {
  xt::Graph g;
};
