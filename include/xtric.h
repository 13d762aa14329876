/*
 * xtric.h — C ABI of the B200-native exact triangle counter (libxtb200.so).
 *
 * Every entry point takes plain pointers and sizes; no C++ or torch types
 * cross this boundary. Host pointers are copied in; the library owns the
 * device memory it allocates. One context = one device + one CUDA stream;
 * calls on one context are serialised by the caller (the reference engine is
 * single-threaded too, main.cpp:53-70). Nothing here aborts the process:
 * every failure is a status code, and xt_last_error() has the detail.
 *
 * Each declaration names the reference interface (sg0/xxtric, file:line) it
 * replaces. Counts are exact int64: a triangle {a,b,c} is counted once in the
 * global count and credited to each of a, b and c in per-vertex counts (the
 * convention of cugraph/cug_triangle_count.py:33-41).
 */
#ifndef XTRIC_H
#define XTRIC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  XT_OK = 0,
  XT_ERR_INVALID = 1,   /* bad argument: null pointer, negative size, id outside [0,nv) */
  XT_ERR_CUDA = 2,      /* CUDA runtime or launch error */
  XT_ERR_OOM = 3,       /* a device allocation failed */
  XT_ERR_IO = 4,        /* file missing, short or with an inconsistent header */
  XT_ERR_OVERFLOW = 5,  /* sizes outside the supported range (nv >= 2^31, ...) */
  XT_ERR_TIMEOUT = 6,   /* a bounded device-side wait gave up */
  XT_ERR_ADMISSION = 7, /* serving: the request can never fit the memory budget */
  XT_ERR_NOT_READY = 8, /* serving: the result is not available yet */
  XT_ERR_NO_DEVICE = 9, /* no CUDA device, or not an sm_100 device */
  XT_ERR_CLOSED = 10    /* serving: the server is closed */
} xt_status;

/* Orientation of each undirected edge {a,b}: from the lower to the higher
 * rank. XT_ORIENT_ID ranks by vertex id, the reference's precedence
 * (u < v < w, xxtric.hpp:165, image/distributed-counting-precedence.png).
 * XT_ORIENT_DEGREE ranks by (degree, id); the global count is identical. */
typedef enum { XT_ORIENT_ID = 0, XT_ORIENT_DEGREE = 1 } xt_orient;

/* lane-tier intersection kinds (xt_graph_set_lane_intersect) */
typedef enum { XT_LANE_BSEARCH = 0, XT_LANE_MERGE = 1 } xt_lane_intersect;

/* xt_graph_from_csr flag: the CSR is already canonical (rows sorted, no
 * duplicates, symmetric, no self loops), the contract under which the
 * reference reads vite files (graph.hpp:294-395), so deduplication is skipped.
 * The reference trusts that contract; here one device pass checks it (rows
 * strictly ascending without their own id, every entry listed back in its
 * partner's row) and the build returns XT_ERR_INVALID before using a row
 * that breaks it. Without the flag the rows are canonicalised on the device
 * first. */
#define XT_CSR_CANONICAL 1

typedef struct xt_ctx xt_ctx;
typedef struct xt_graph xt_graph;

typedef struct {
  int64_t nv;             /* vertices */
  int64_t n_input;        /* input entries (directed CSR entries or edge-list rows) */
  int64_t n_edges;        /* undirected unique non-loop edges == oriented edges |E+| */
  int64_t max_degree;     /* max undirected degree */
  int64_t max_out_degree; /* max d+ after orientation */
  int64_t max_in_degree;  /* max d- after orientation */
  int64_t wedge_work;     /* sum over oriented (u,v) of d+(v): items a tail-grouped count streams */
  int64_t stream_work;    /* sum over u of C(d+(u),2): candidate columns this count streams (the
                             suffix of N+(u) after each out-neighbour) */
  int64_t alg_bytes;      /* bytes the count's loads request, repeats included (a suffix streamed by
                             several heads counts each time; L2 serves many of the repeats):
                             16(nv+1) offsets + 4|E+| member columns + 8|E+| in-records +
                             4 stream_work candidate columns */
  int64_t tail_alg_bytes; /* the tail-grouped figure: 8(nv+1) + 4|E+| + sum (16 + 4 d+(v)) */
  int32_t orient;         /* xt_orient used */
  int32_t reserved;
  int64_t footprint_bytes; /* bytes of the arrays the count reads, each counted once: offsets and
                              in-record offsets 16(nv+1), columns 4|E+|, padded columns, in-records
                              8|E+|: the DRAM traffic of a count that never re-reads */
  int64_t cluster_tasks;   /* global count: the tasks of its thread-block cluster tier (see
                              xt_graph_set_cluster); 0 when no head needs it */
} xt_graph_info;

/* ---- context ------------------------------------------------------------
 * Replaces the device set-up of TriangleCountingSingle's constructor
 * (xxtric-gpu.hpp:40-44), which hard-codes device 0. */
xt_status xt_open(int device, xt_ctx **out);
xt_status xt_close(xt_ctx *ctx);
/* use an existing cudaStream_t (passed as void*) instead of the context's own */
xt_status xt_set_stream(xt_ctx *ctx, void *cuda_stream);
/* wait for all work queued on the context's stream (the generators and
 * xt_count_async return before their kernels finish) */
xt_status xt_synchronize(xt_ctx *ctx);
const char *xt_strerror(xt_status s);
const char *xt_last_error(const xt_ctx *ctx);
/* test hook: make the k-th device allocation from now fail (k<=0 disarms) */
xt_status xt_debug_fail_alloc(xt_ctx *ctx, int64_t k);
/* number of this library's own kernels launched on the context so far
 * (library sorts and scans from CUB are not included) */
int64_t xt_launch_count(const xt_ctx *ctx);
/* device bytes this context's own allocations hold now (live) and at most
 * since it opened or since the last reset (peak); reset_peak != 0 restarts
 * the high-water mark at the live figure. No counterpart in the reference. */
xt_status xt_mem_stats(xt_ctx *ctx, int64_t *live, int64_t *peak, int reset_peak);

/* ---- graph build ---------------------------------------------------------
 * Replaces TriangleCountingSingle(Graph*) (xxtric-gpu.hpp:27-156): host CSR in
 * the vite layout of Graph (graph.hpp:52-275; offsets int64[nv+1], tails
 * int64[offsets[nv]]) is copied to the device and turned into an oriented
 * int32-column / int64-offset CSR there. */
xt_status xt_graph_from_csr(xt_ctx *ctx, int64_t nv, const int64_t *offsets, const int64_t *tails, int flags,
                            int orient, xt_graph **out);
/* the same from a host edge list of ne (src,dst) rows with int32 ids; rows
 * may repeat, appear in one direction only or be self loops */
xt_status xt_graph_from_edges(xt_ctx *ctx, int64_t nv, int64_t ne, const int32_t *src, const int32_t *dst,
                              int orient, xt_graph **out);
/* the same from int32 edge lists already in device memory (not freed) */
xt_status xt_graph_from_device_edges(xt_ctx *ctx, int64_t nv, int64_t ne, const int32_t *d_src,
                                     const int32_t *d_dst, int orient, xt_graph **out);
/* Replaces BinaryEdgeList::read (graph.hpp:294-395) followed by the
 * TriangleCountingSingle constructor: the vite file at path (elem_bytes 8, or
 * 4 for USE_32_BIT_GRAPH) is streamed through pinned staging buffers to the
 * device, whose kernels take the tails out of the {tail, weight} records, and
 * built like xt_graph_from_csr (flags: XT_CSR_CANONICAL or 0). The host never
 * touches a record. XT_ERR_IO for a file whose size does not match its header
 * or whose offsets do not start at 0 and end at ne. */
xt_status xt_graph_from_vite(xt_ctx *ctx, const char *path, int elem_bytes, int flags, int orient,
                             xt_graph **out);
xt_status xt_graph_get_info(const xt_graph *g, xt_graph_info *info);
/* copy the oriented CSR out (host buffers of nv+1 and n_edges entries), in
 * the library's internal numbering: vertices renumbered by orientation rank,
 * so every row holds only higher ids, ascending */
xt_status xt_graph_get_csr(const xt_graph *g, int64_t *offsets, int32_t *cols);
/* internal id -> input id (host buffer of nv entries) */
xt_status xt_graph_get_perm(const xt_graph *g, int32_t *new_to_old);
/* Replaces TriangleCountingSingle::clear() (xxtric-gpu.hpp:272-285). */
xt_status xt_graph_free(xt_graph *g);

/* ---- counting ------------------------------------------------------------
 * Replaces TriangleCountingSingle::count() (xxtric-gpu.hpp:192-270): the
 * global count, and per-vertex counts into a host array of nv entries when
 * per_vertex is not null. Synchronous, like the reference. */
xt_status xt_count(xt_graph *g, int64_t *global, int64_t *per_vertex);
/* the same into device memory, asynchronous on the context stream;
 * d_per_vertex (nullable) holds nv int64 entries and is overwritten */
xt_status xt_count_async(xt_graph *g, int64_t *d_global, int64_t *d_per_vertex);

/* No counterpart in the reference (its per-edge work is internal): the
 * global count and, for every oriented edge, the number of triangles that
 * contain it (its k-truss support), into a host array of n_edges entries in
 * the order of xt_graph_get_csr (internal numbering; xt_graph_get_perm maps
 * ids back). The supports sum to 3 x global. Synchronous. */
xt_status xt_count_edges(xt_graph *g, int64_t *global, int64_t *support);
/* the same into device memory, asynchronous on the context stream;
 * d_support holds n_edges int64 entries and is overwritten */
xt_status xt_count_edges_async(xt_graph *g, int64_t *d_global, int64_t *d_support);

/* ---- edge-sharded counting over several GPUs -------------------------------
 * Replace the per-GPU share of the reference's multi-GPU count
 * (TriangleCounting::count, xxtric-gpu-vmm-mpi.hpp:89-129: every GPU counts
 * its part, then MPI_Reduce sums the parts on rank 0). Here every GPU holds
 * the whole graph (one process per GPU, each built from the same input) and
 * counts one shard of the count's schedule: the tasks of every tier (CTA,
 * warp and lane tasks, cluster tasks) whose index is shard modulo nshards.
 * Every triangle falls in exactly one task, so the nshards shards' global
 * counts, per-vertex counts and per-edge supports each sum to those of
 * xt_count / xt_count_edges; a caller sums them with one all-reduce
 * (xxtric_b200.shards does it over NCCL). Asynchronous on the context
 * stream, device outputs overwritten with the shard's part (d_per_vertex:
 * nv int64, nullable; d_support: n_edges int64 in xt_graph_get_csr order).
 * XT_ERR_INVALID unless 0 <= shard < nshards. */
xt_status xt_count_shard_async(xt_graph *g, int shard, int nshards, int64_t *d_global, int64_t *d_per_vertex);
xt_status xt_count_edges_shard_async(xt_graph *g, int shard, int nshards, int64_t *d_global, int64_t *d_support);

/* Replaces the kernel launcher single_gpu_count(nv, d_indices, d_edge_list,
 * d_local_count) (counting.cuh:259-265, counting.cu:537-577): the reference's
 * device CSR (int64 offsets, int64 tails; rows sorted, deduped, symmetric)
 * is oriented and counted on the given stream. Unlike the reference, which
 * accumulates into a caller-zeroed counter and reports nothing, this
 * overwrites *d_count (accumulate != 0 adds instead) and returns errors;
 * rows that break the layout's promise are rejected with XT_ERR_INVALID (see
 * XT_CSR_CANONICAL) and *d_count is left as it was.
 * Scratch memory is allocated stream-ordered and released before return. */
xt_status xt_count_device(int64_t nv, const int64_t *d_indices, const int64_t *d_edge_list, int64_t *d_count,
                          int accumulate, void *cuda_stream);

/* No counterpart in the reference. The count of the same device CSR as
 * xt_count_device (int64 offsets, int64 tails; rows sorted ascending without
 * repeats or self loops, symmetric: this entry cannot sort, so it checks and
 * rejects other rows), for callers that cannot allocate device memory while they run:
 * it calls no cudaMalloc, cudaFree or other allocating routine. Its scratch is
 * one fixed 64 MiB array inside the library, present on every GPU that loads
 * the library until the process exits; it holds 8 bytes per vertex, so
 * nv must not exceed 8,389,088 (else XT_ERR_OVERFLOW). The first call on a
 * device sets up the array's address (make it before any stream capture).
 * Calls that overlap on one device race on the shared array: serialise them.
 * Orientation is by vertex id. Overwrites *d_count, or adds to it when
 * accumulate != 0; XT_ERR_INVALID when an offset is negative or decreases, a
 * row is out of order, repeats an id, holds its own id or an id outside
 * [0, nv), or an edge is listed in one of its two rows only (input not
 * symmetric, in either direction); on any error *d_count keeps its value.
 * XT_ERR_CUDA, before anything is launched, when a CUDA error from earlier
 * work is still pending (it is left for the caller to read). Synchronises the
 * given stream before returning. */
xt_status xt_count_device_static(int64_t nv, const int64_t *d_indices, const int64_t *d_edge_list,
                                 int64_t *d_count, int accumulate, void *cuda_stream);

/* ---- batching form ---------------------------------------------------------
 * No counterpart in the reference, which counts one graph per run. Many
 * independent graphs become one graph object: graph g has the vertices
 * [vertex_offsets[g], vertex_offsets[g+1]) and the edge rows
 * [edge_offsets[g], edge_offsets[g+1]) of src/dst, whose ids are LOCAL to
 * their graph (0 .. n_g - 1). One build serves all graphs and one count
 * launch covers them all; xt_count_groups returns every graph's own count,
 * identical to counting that graph alone. */
xt_status xt_graph_from_batch(xt_ctx *ctx, int64_t n_graphs, const int64_t *vertex_offsets,
                              const int64_t *edge_offsets, const int32_t *src, const int32_t *dst, int orient,
                              xt_graph **out);
/* the same with src/dst in device memory (offset tables on the host) */
xt_status xt_graph_from_device_batch(xt_ctx *ctx, int64_t n_graphs, const int64_t *vertex_offsets,
                                     const int64_t *edge_offsets, const int32_t *d_src, const int32_t *d_dst,
                                     int orient, xt_graph **out);
/* One call: builds the batch (host buffers, as xt_graph_from_batch), counts
 * it once and frees it; *total and per_graph (n_graphs entries, nullable)
 * receive the counts. */
xt_status xt_batch_count(xt_ctx *ctx, int64_t n_graphs, const int64_t *vertex_offsets, const int64_t *edge_offsets,
                         const int32_t *src, const int32_t *dst, int orient, int64_t *total, int64_t *per_graph);
/* graphs in a batch (0 for a single graph) */
int64_t xt_graph_groups(const xt_graph *g);
/* total and per-graph counts (host buffer of xt_graph_groups entries, nullable) */
xt_status xt_count_groups(xt_graph *g, int64_t *total, int64_t *per_group);
xt_status xt_count_groups_async(xt_graph *g, int64_t *d_total, int64_t *d_per_group);
/* Capture the graph's count (its memsets and its one persistent launch) into
 * a CUDA graph once; xt_count_groups then replays it. */
xt_status xt_graph_capture(xt_graph *g);
/* Schedule thresholds (0 = automatic): items per CTA task, the work limit of
 * a warp task, and the largest member id range kept as a bitmap (beyond it a
 * hash). Re-plans (and re-captures a captured graph). */
xt_status xt_graph_set_tuning(xt_graph *g, int64_t block_work, int64_t warp_work, int64_t bitmap_bits);
/* Tier limits: heads with at most lane_work candidates are counted one per
 * lane (binary search in the row), heads with at most warp_work candidates
 * and at most 256 members one per warp, the rest by CTA tasks. Negative =
 * automatic (the lane tier is on only for graphs of 2^30 or more
 * candidates), 0 = tier off. Re-plans (and re-captures a captured graph). */
xt_status xt_graph_set_tiers(xt_graph *g, int64_t lane_work, int64_t warp_work);
/* Global count: a bulk L2 prefetch of each in-record's suffix one record
 * batch ahead (on != 0) or none (0, the default). It pays on graphs whose
 * suffixes are seldom re-read from L2 (many small graphs in one batch) and
 * costs issue slots on graphs whose suffixes are; the autotuner tries both.
 * Re-captures a captured graph. */
xt_status xt_graph_set_prefetch(xt_graph *g, int on);
/* Global count, cluster tier: with on != 0 a head with more out-neighbours
 * than one CTA's member set holds (2,048; the id orientation gives hubs
 * many) is counted by a thread-block cluster of 8 CTAs whose shared
 * memories hold up to 16,384 of them between them, each candidate looked up
 * in the table of the CTA whose id range holds it through distributed
 * shared memory, and the cluster's counts summed there. With 0 (the
 * default) such a head is counted by CTA tasks over parts of 2,048 members,
 * each streaming all of its in-records: on the B200 that is the faster of
 * the two (Chung-Lu n=4.19M under the id orientation: 343 ms against 704 ms
 * with clusters), because a lookup in another CTA's shared memory costs far
 * more than the re-streamed candidates it saves. The reference's
 * counterpart is the cluster kernel of counting.cu:1043-1143
 * (cluster.map_shared_rank reduction). The per-vertex and per-edge counts
 * always use the CTA parts. Counts are identical either way. Re-plans (and
 * re-captures a captured graph). */
xt_status xt_graph_set_cluster(xt_graph *g, int on);
/* Lane tier intersection (heads counted one per lane, see
 * xt_graph_set_tiers): each candidate of an in-record's suffix is found in
 * N+(v) from the position after the previous one, by binary search
 * (XT_LANE_BSEARCH, the default) or by stepping forward, a two-pointer merge
 * of the two ascending lists (XT_LANE_MERGE), cheaper when N+(v) is short
 * next to the suffixes. The binary search is the reference's own
 * (count_if_edge_exists, counting.cu:95-131; check_edgelist,
 * xxtric.hpp:516-588); the reference has no merge. The autotuner tries both
 * where the plan has lane tasks. Counts are identical. Re-captures a
 * captured graph. */
xt_status xt_graph_set_lane_intersect(xt_graph *g, int kind);
/* No counterpart in the reference (its kernels take vertices by grid
 * index): warp tasks, and lane tasks in groups of 32 heads, are taken from
 * their global cursor `claim` at a time (1..64; 0, the default: 4 for a
 * graph built as a batch, 1 otherwise). One atomic on one address per task
 * limits schedules of many small tasks (the 4,096-graph batch: 38.2 ms a
 * count with 1, 30.4 ms with 4); larger blocks leave a longer tail on
 * graphs whose warp tasks are fewer (R-MAT scale 22: 4.69 ms with 1, 4.79
 * with 4). The autotuner tries 1, 4 and 16. Counts are identical.
 * Re-captures a captured graph. */
xt_status xt_graph_set_claim(xt_graph *g, int claim);
/* Test hook, no counterpart in the reference: caps the eviction chain of the
 * global count's cuckoo member sets at `iters` steps (negative: the default
 * of 64). With 0 or 1 nearly every hashed set falls back to linear probing,
 * which lets a test reach that path; counts are unchanged. */
xt_status xt_graph_debug_cuckoo_iters(xt_graph *g, int iters);
/* Autotuner: a coordinate search of the three thresholds, then the suffix
 * prefetch on and off, the lane tier's merge and the claim block
 * (xt_graph_set_claim), timing `reps` counts each, keeping the fastest; with
 * cache_path it first looks the
 * (GPU, graph class) key up in that text file and appends new results.
 * A JSON report of the trials goes to report (nullable). */
xt_status xt_graph_autotune(xt_graph *g, int reps, const char *cache_path, char *report, int64_t report_len);

/* The batch workload of this repository's benchmarks: for graph i of
 * n_graphs, kind (0 = unit-square random geometric graph, 1 = Erdos-Renyi
 * G(n, m)), vertex count (log-uniform in [256, 65536)), mean degree
 * (log-uniform in [8, 64)) and its own seed, all derived from seed. */
xt_status xt_batch_spec(int64_t n_graphs, uint64_t seed, int32_t *kind, int64_t *n, double *mean_deg,
                        uint64_t *graph_seed);
/* Generates those graphs on the device: local-id edge rows (random geometric:
 * every pair u < v within distance sqrt(mean_deg / (pi n)); Erdos-Renyi:
 * round(n mean_deg / 2) uniform pairs), edge_offsets (host, n_graphs + 1)
 * filled, the arrays allocated by the library (release with xt_device_free). */
xt_status xt_gen_batch(xt_ctx *ctx, int64_t n_graphs, const int32_t *kind, const int64_t *n, const double *mean_deg,
                       const uint64_t *graph_seed, int64_t *edge_offsets, int32_t **d_src, int32_t **d_dst);
xt_status xt_device_free(xt_ctx *ctx, void *p);

/* ---- serving form -----------------------------------------------------------
 * No counterpart in the reference, which counts one graph per process run.
 * A server owns `slots` contexts (one CUDA stream and one host worker thread
 * each) on one device. Count queries (host edge lists, graph-local int32
 * ids) are admitted against a device-memory budget: each query's build and
 * count hold at most xt_serve_estimate(nv, ne) bytes, and the queries in
 * flight never hold more than the budget between them. Whenever a slot is
 * free it takes every queued query that fits (first come first served, up to
 * max_batch_graphs / max_batch_edges), builds them on the device as one
 * batch and counts them in one launch; queries that arrive meanwhile wait
 * only for the next free slot, and the slots' batches overlap on the device.
 * Each query's count equals the count of its graph alone (xt_count). */
typedef struct xt_server xt_server;
typedef struct {
  int64_t budget_bytes;     /* device bytes for queries in flight; <= 0: 150 GiB. Capped at the
                               device's free memory at open, less 2 GiB */
  int64_t max_batch_graphs; /* queries per batch, at most; <= 0: 4096 */
  int64_t max_batch_edges;  /* edge rows per batch, at most (a larger query runs alone); <= 0: 2^26 */
  int32_t slots;            /* batches in flight at once; <= 0: 3 */
  int32_t orient;           /* xt_orient of every query */
} xt_serve_config;
typedef struct {
  int64_t budget_bytes;     /* the budget in force */
  int64_t submitted, completed, failed, rejected;
  int64_t queued;           /* waiting for a slot */
  int64_t in_flight;        /* admitted, result not yet published */
  int64_t batches;          /* batches run */
  int64_t max_batch;        /* most queries in one batch */
  int64_t budget_used;      /* estimated bytes held by queries in flight now */
  int64_t budget_peak;      /* ... and at most */
  int64_t device_peak;      /* measured device bytes the slots' allocations held at most at once */
  int64_t launches;         /* this library's kernels launched by the server */
} xt_serve_stats;
/* device bytes one query of nv vertices and ne edge rows may hold while it
 * is built and counted (alone or in a batch: batch figures add up) */
int64_t xt_serve_estimate(int64_t nv, int64_t ne);
xt_status xt_serve_open(int device, const xt_serve_config *cfg, xt_server **out);
/* Queues a count of the graph with nv vertices and ne rows (src[i], dst[i])
 * (ids in [0, nv); rows may repeat or be loops). The buffers are read
 * while the query runs: keep them unchanged until its result is taken
 * (pinned host memory copies fastest). XT_ERR_ADMISSION when the query
 * alone exceeds the budget, XT_ERR_CLOSED after xt_serve_close began. */
xt_status xt_serve_submit(xt_server *srv, int64_t nv, int64_t ne, const int32_t *src, const int32_t *dst,
                          int64_t *ticket);
/* The query's result: XT_ERR_NOT_READY while it runs; otherwise its status
 * (XT_OK with *count, or the error that failed it, e.g. XT_ERR_INVALID for
 * an id outside [0, nv)) and the seconds from submit to result
 * (latency_s, nullable). A result is returned once: the ticket is then
 * forgotten (XT_ERR_INVALID afterwards). */
xt_status xt_serve_poll(xt_server *srv, int64_t ticket, int64_t *count, double *latency_s);
/* xt_serve_poll that blocks up to timeout_ms (< 0: no limit); XT_ERR_TIMEOUT
 * when the result is still not there */
xt_status xt_serve_wait(xt_server *srv, int64_t ticket, int64_t timeout_ms, int64_t *count, double *latency_s);
xt_status xt_serve_get_stats(xt_server *srv, xt_serve_stats *stats);
/* one batch the server ran: times in ns since xt_serve_open (taken from the
 * queue, built and planned, results published) */
typedef struct {
  int64_t t_take_ns, t_built_ns, t_done_ns;
  int64_t graphs, edge_rows;
  int32_t slot;
  int32_t status; /* xt_status of the batch (per-query retries not shown) */
} xt_serve_batch;
/* copies the most recent min(max, n) batch records (the server keeps the
 * last 65,536) into out, oldest first; returns how many, or -1 */
int64_t xt_serve_batches(xt_server *srv, xt_serve_batch *out, int64_t max);
/* Stops admitting, fails the queued queries with XT_ERR_CLOSED, lets the
 * batches in flight finish, joins the workers and frees everything; results
 * not yet taken are lost. No other call on this server may run during or
 * after it (a thread still waiting in xt_serve_wait must return first). */
xt_status xt_serve_close(xt_server *srv);

/* ---- synthetic inputs on the device --------------------------------------
 * Deterministic counter-based generators (same bits for the same seed on any
 * GPU and in the CPU oracle). Outputs are device int32 arrays of ne rows. */
/* R-MAT: 2^scale vertices, quadrant weights in 1/65536 units, +-noise_pct %
 * multiplicative noise per edge and level, ids permuted when permute != 0 */
xt_status xt_gen_rmat(xt_ctx *ctx, int scale, int64_t ne, uint64_t seed, int a16, int b16, int c16,
                      int noise_pct, int permute, int32_t *d_src, int32_t *d_dst);
/* Chung-Lu from a host integer CDF of n+1 entries (see xt_chunglu_cdf) */
xt_status xt_gen_chunglu(xt_ctx *ctx, int64_t n, const uint64_t *cdf, int64_t ne, uint64_t seed, int permute,
                         int32_t *d_src, int32_t *d_dst);
/* Chung-Lu integer weight CDF (host): n+1 entries; returns the edge count */
int64_t xt_chunglu_cdf(int64_t n, double gamma, double mean_deg, double max_deg, uint64_t *cdf);
/* Erdos-Renyi G(n, ne): uniform ordered pairs */
xt_status xt_gen_er(xt_ctx *ctx, int64_t n, int64_t ne, uint64_t seed, int32_t *d_src, int32_t *d_dst);
/* Replaces the loops of GenerateRGG(nv).generate (graph.hpp:745-1364) and
 * its LCG (utils.hpp:245-430) for the -n path without random edges (-p 0):
 * the reference's random geometric graph as nprocs strip ranks build it,
 * generated on the device, bit for bit the edge set of xt_rgg_generate.
 * radius <= 0 selects the reference's r(n) (graph.hpp:788-791). Writes each
 * undirected edge once, as (a, b) with a < b, into d_src/d_dst (device
 * int32 arrays of cap rows) and its count into *n_pairs; with d_src == NULL
 * only *n_pairs is filled (sizing call). XT_ERR_OVERFLOW when cap is short. */
xt_status xt_gen_rgg(xt_ctx *ctx, int64_t nv, int nprocs, double radius, int64_t cap, int64_t *n_pairs,
                     int32_t *d_src, int32_t *d_dst);
/* The same graph generated and built on the device in one call (the -n path
 * of main.cpp:90-91 followed by the TriangleCountingSingle constructor); the
 * library holds every buffer. n_input of its info is the reference's
 * directed entry count, twice the pairs. */
xt_status xt_graph_from_rgg(xt_ctx *ctx, int64_t nv, int nprocs, double radius, int orient, xt_graph **out);

/* ---- host-side graph input (no device needed) ------------------------------ */

/* Replaces BinaryEdgeList::read (graph.hpp:294-395) for one process: the vite
 * binary layout [nv][ne][offsets: nv+1][ne x {tail, weight}] with 8-byte
 * fields (elem_bytes 8, the default GraphElem/GraphWeight of deftypes.hpp:
 * 45-49) or 4-byte fields (elem_bytes 4, USE_32_BIT_GRAPH, deftypes.hpp:40-44).
 * With offsets == NULL only *nv and *ne are filled (sizing call). The file
 * size must match the header exactly; weights are skipped. */
xt_status xt_vite_read(const char *path, int elem_bytes, int64_t *nv, int64_t *ne, int64_t *offsets,
                       int64_t *tails);
/* writes the same layout with unit weights */
xt_status xt_vite_write(const char *path, int elem_bytes, int64_t nv, const int64_t *offsets,
                        const int64_t *tails);

/* Tab-separated edge list, the input of the reference's cuGraph comparison
 * (cugraph/cug_triangle_count.py:23-26: src, dst, optional weight; ids as
 * given, so *nv = largest id + 1). With src == NULL only *nv and *ne are
 * filled (sizing call); otherwise up to cap rows go to src/dst
 * (XT_ERR_OVERFLOW beyond cap). '#'/'%' comment and blank lines are skipped;
 * a malformed line is XT_ERR_IO. */
xt_status xt_tsv_read(const char *path, int64_t *nv, int64_t *ne, int32_t *src, int32_t *dst, int64_t cap);
/* writes ne rows "src<TAB>dst<TAB>1" */
xt_status xt_tsv_write(const char *path, int64_t ne, const int32_t *src, const int32_t *dst);

/* Replaces GenerateRGG(nv).generate(LCG, unit weights, random_edge_pct)
 * (graph.hpp:745-1364, utils.hpp:245-430; main.cpp:90-91) as nprocs strip
 * ranks would build it under mpiexec -n nprocs (the graph depends on the rank
 * count). radius <= 0 selects the reference's r(n) (graph.hpp:788-791).
 * random_edge_pct in [0,100) adds the reference's extra random edges, drawn
 * from seed. Rows are sorted; with offsets == NULL only *ne is filled. */
xt_status xt_rgg_generate(int64_t nv, int nprocs, double radius, double random_edge_pct, uint64_t seed,
                          int64_t cap, int64_t *ne, int64_t *offsets, int64_t *tails);

#ifdef __cplusplus
}
#endif
#endif /* XTRIC_H */
