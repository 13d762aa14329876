// Degree-binned schedule and the exact triangle-count kernel.
//
// Vertices are numbered by orientation rank (see build.cu), so every triangle
// {u,v,w} with u < v < w is the edges u->v, u->w, v->w. The reference finds it
// from the lowest corner i=u: for every pair m < n of its sorted row it
// binary-searches adj(v) for w (xxtric.hpp:150-207, check_edgelist
// xxtric.hpp:516-545). Here it is found from the MIDDLE corner v:
//   1. N+(v) is loaded once into shared memory as a membership structure:
//      a bitmap over the words spanning [min N+(v), max N+(v)] when that range
//      is small enough, else an open-addressing hash table over the whole
//      region (load factor <= 1/4);
//   2. for every in-edge u->v, the suffix of N+(u) after v (the reference's
//      n > m range) is streamed through it; candidates outside
//      [min N+(v), max N+(v)] fail the test at once (the reference's
//      edge_above_min / edge_within_max prunes, xxtric.hpp:576-588).
// Items streamed: sum over u of C(d+(u), 2), each tested in shared memory.
//
// Schedule (make_plan): per head v, work(v) = total suffix length.
//   lane tier: work(v) <= tiny_work -> one lane per head, members
//              binary-searched in the row itself
//   warp tier: d+(v) <= kWarpDmax and work(v) <= warp_work -> one warp per
//              head, member set in the warp's slice of shared memory
//   CTA tier : otherwise -> CTA tasks over chunks of v's in-records of about
//              block_work items; N+(v) beyond kBlockDmax members is split
//              into parts, one task per (part, chunk)
// One persistent kernel drains the CTA tasks first (the large ones), then the
// warp tasks, then the lane tasks, each from its own global atomic cursor.
// Inside a task, lanes walk whole suffixes in aligned 32-byte pairs of the
// padded column array, with no masking (see stream_kind).
#include <cooperative_groups.h>
#include <type_traits>
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/transform_iterator.h>

#include "xt_internal.cuh"

namespace xt {

// Tuning constants (compile-time; the XT_* macros let a build override them)
#ifndef XT_THREADS
#define XT_THREADS 256
#endif
// CTA tasks of up to 2^17 candidates, warp tasks of up to 4,096 (8,192 on
// graphs of 2^34 or more candidates): swept with the cuckoo member sets
// (R-MAT s24 / s22 / Chung-Lu 27.32 / 4.70 / 7.99 ms at 2^17 and 8,192
// against 28.09 / 4.99 / 8.39 at 2^16 and 4,096; at 2^17, 4,096 gave 27.69 /
// 4.72 / 7.97; 2^18 28.52 ms at s24; 32,768 9.49 ms on Chung-Lu). On small
// graphs the larger warp limit moves heads onto warp tasks, which run last
// and leave a tail: R-MAT s18 0.195 -> 0.35 ms with 8,192.
#ifndef XT_BLOCK_WORK_LOG2
#define XT_BLOCK_WORK_LOG2 17
#endif
#ifndef XT_WARP_WORK
#define XT_WARP_WORK 4096
#endif
#ifndef XT_WARP_WORK_LARGE
#define XT_WARP_WORK_LARGE 8192
#endif
constexpr int kThreads = XT_THREADS;
constexpr int kWarps = kThreads / 32;
#ifndef XT_MIN_BLOCKS
#define XT_MIN_BLOCKS 4
#endif
// CTAs per SM the register budget is sized for: 4 x 256 threads leave 64
// registers a thread (no spills). Swept with the task size at R-MAT s24
// (before the cuckoo sets): 3 CTAs/SM with 2^17-candidate tasks 34.2 ms, 4
// with 2^17 33.8 ms, 4 with 2^16 32.1 ms, 4 with 2^15 35.1 ms, 5 (spilling)
// 53.9 ms
constexpr int kMinBlocks = XT_MIN_BLOCKS;
constexpr int kBlockWords = 8192;  // CTA region: 8192-slot hash or 2^18-bit bitmap
// warp tasks run after the CTA tasks and split the CTA region among the warps
constexpr int kWarpWords = kBlockWords / kWarps;  // 1024: a 1024-slot hash or a 32K-bit bitmap
constexpr int kWarpDmax = kWarpWords / 4;         // hash load factor <= 1/4
constexpr int64_t kWarpWork = XT_WARP_WORK;
#ifndef XT_BLOCK_DMAX
#define XT_BLOCK_DMAX 2048
#endif
constexpr int kBlockDmax = XT_BLOCK_DMAX;
// the warps' member counters share the CTA's
static_assert(kWarps * kWarpDmax <= kBlockDmax, "warp member counters exceed the CTA's");
// Cluster tier (global count): a head whose members overflow a CTA's set
// (more than kBlockDmax, as the id orientation gives hubs) is counted by a
// cluster of kCluster CTAs holding up to kClusterDmax members per part
constexpr int kCluster = 8;
constexpr int kClusterDmax = kCluster * kBlockDmax;
constexpr int64_t kBlockWorkMin = int64_t(1) << 14;
constexpr int64_t kBlockWorkMax = int64_t(1) << XT_BLOCK_WORK_LOG2;

// Run-time schedule thresholds (the binning of make_plan).
struct PlanParams {
  int64_t tiny_work;   // a head with at most this much work is a lane task
  int64_t warp_work;   // ... else one with d+(v) <= warp_dmax and at most this much work is a warp task
  int64_t block_work;  // items per CTA task
  int32_t warp_dmax;
  int32_t batches_per_warp;  // CTA task: record batches per warp, at least
  int32_t lane_pairs;        // CTA task: pairs per lane on an average record, at least
};
#ifndef XT_BATCHES_PER_WARP
#define XT_BATCHES_PER_WARP 4
#endif
// graphs of 2^34 or more candidates: more, smaller record batches per CTA
// task (R-MAT s24 27.26 ms with 4, 26.47 with 5, 26.79 with 6, 27.59 with 8;
// at 6, s22 and Chung-Lu were 0.5% slower, so smaller graphs keep 4)
#ifndef XT_BATCHES_PER_WARP_LARGE
#define XT_BATCHES_PER_WARP_LARGE 5
#endif
#ifndef XT_LANE_PAIRS
#define XT_LANE_PAIRS 2
#endif
#ifndef XT_TINY_WORK
#define XT_TINY_WORK 32
#endif
// global count: warp tasks keep hashed member sets as cuckoo tables (two
// slots per id, branch-free probes) and reset only the slots they filled
#ifndef XT_WARP_CUCKOO
#define XT_WARP_CUCKOO 1
#endif
// streaming: L2 prefetch of the pair XT_PF_DIST steps ahead (0: none;
// measured slower: the kernel is issue-bound, R-MAT s24 28.55 -> 30.4 ms at
// distance 2)
#ifndef XT_PF_DIST
#define XT_PF_DIST 0
#endif
// per-vertex mode: bitmap hits credited without a branch
#ifndef XT_PV_PRED
#define XT_PV_PRED 1
#endif
#ifndef XT_LANE_LOOP
#define XT_LANE_LOOP 0
#endif
constexpr bool kWarpCuckoo = XT_WARP_CUCKOO != 0;
// bit of the context's error word set when a bounded staging wait gave up
constexpr int kErrStageTimeout = 8;
constexpr int32_t kEmpty = -1;

// A warp or CTA task: the in-records [k0, k0 + nrec) of head v streamed
// through the members col[r0, r0 + nmem), 2^lg_s lanes per record.
struct __align__(16) Task {
  int64_t k0;
  int64_t r0;
  int32_t v;
  int32_t nrec;
  int32_t nmem;
  int32_t lg_s;
};

struct Plan {
  int64_t n_btask = 0;         // CTA tasks
  Task *d_bt = nullptr;
  int64_t n_wtask = 0;         // warp tasks
  Task *d_wt = nullptr;
  int64_t n_ttask = 0;         // lane tasks: one head per lane
  int32_t *d_tt = nullptr;
  unsigned long long *d_cursor = nullptr;  // [0] CTA, [1] warp, [2] lane, [3] cluster task cursors
  int64_t n_ctask = 0;         // cluster tasks (global count)
  Task *d_ct = nullptr;
  int64_t n_btask0 = 0;        // the CTA tasks of the other heads, which the global count
  Task *d_bt0 = nullptr;       //   runs beside the cluster tasks
  int grid_global = 0, grid_pv = 0, grid_es = 0, grid_cluster = 0;
  int64_t block_work = 0, warp_work = 0;   // the thresholds the plan was made with
  int64_t bitmap_bits = 0;
};

static unsigned grid_for(int64_t n, int block, int sm_count) {
  int64_t g = (n + block - 1) / block;
  int64_t cap = int64_t(sm_count) * 32;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (unsigned)g;
}

#define XT_GRID_STRIDE(i, n) \
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < (n); i += int64_t(gridDim.x) * blockDim.x)

// ---- plan kernels -----------------------------------------------------------

// in-record e's candidates (its suffix length), 0 past the last record: the
// input of the plan's prefix sum, read straight from the records
struct RecLen {
  const InRec *rec;
  int64_t ne;
  __host__ __device__ int64_t operator()(int64_t e) const { return e < ne ? int64_t(rec_len(rec[e])) : 0; }
};

// Graph statistics in one pass over the vertices: st[0] the largest degree
// (out + in), st[1] the largest out-degree, st[2] the largest in-degree,
// st[3] the tail-grouped work sum over edges u->v of d+(v) = sum over v of
// d-(v) d+(v)
__global__ void k_vertex_stats(const int64_t *__restrict__ off, const int64_t *__restrict__ ioff, int64_t nv,
                               unsigned long long *__restrict__ st) {
  unsigned long long md = 0, mo = 0, mi = 0, wsum = 0;
  XT_GRID_STRIDE(i, nv) {
    const unsigned long long dout = off[i + 1] - off[i], din = ioff[i + 1] - ioff[i];
    md = max(md, dout + din);
    mo = max(mo, dout);
    mi = max(mi, din);
    wsum += dout * din;
  }
  for (int o = 16; o; o >>= 1) {
    md = max(md, __shfl_xor_sync(0xffffffffu, md, o));
    mo = max(mo, __shfl_xor_sync(0xffffffffu, mo, o));
    mi = max(mi, __shfl_xor_sync(0xffffffffu, mi, o));
    wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&st[0], md);
    atomicMax(&st[1], mo);
    atomicMax(&st[2], mi);
    atomicAdd(&st[3], wsum);
  }
}

// tasks of head v: nb CTA tasks (parts x chunks), nw warp tasks, nt lane tasks (0 or 1 each)
__device__ __forceinline__ void classify(int64_t v, const int64_t *__restrict__ off, const int64_t *__restrict__ ioff,
                                         const int64_t *__restrict__ P, const PlanParams pp, int64_t &nb,
                                         int64_t &nw, int64_t &nt, int64_t &parts, int64_t &chunks, int64_t &work) {
  const int64_t dp = off[v + 1] - off[v];
  const int64_t k0 = ioff[v], k1 = ioff[v + 1];
  nb = nw = nt = parts = chunks = 0;
  work = P[k1] - P[k0];
  if (dp == 0 || work == 0) return;
  if (work <= pp.tiny_work) {
    nt = 1;
    return;
  }
  if (dp <= pp.warp_dmax && work <= pp.warp_work) {
    nw = 1;
    return;
  }
  parts = (dp + kBlockDmax - 1) / kBlockDmax;
  chunks = (work + pp.block_work - 1) / pp.block_work;
  nb = parts * chunks;
}

__global__ void k_plan_count(int64_t nv, const int64_t *__restrict__ off, const int64_t *__restrict__ ioff,
                             const int64_t *__restrict__ P, const PlanParams pp, int64_t *__restrict__ nb_out,
                             int64_t *__restrict__ nw_out, int64_t *__restrict__ nt_out) {
  XT_GRID_STRIDE(v, nv) {
    int64_t nb, nw, nt, parts, chunks, work;
    classify(v, off, ioff, P, pp, nb, nw, nt, parts, chunks, work);
    nb_out[v] = nb;
    nw_out[v] = nw;
    nt_out[v] = nt;
  }
}

// first k in [lo,hi] with P[k] >= x
__device__ __forceinline__ int64_t lower_bound_i64(const int64_t *__restrict__ P, int64_t lo, int64_t hi, int64_t x) {
  while (lo < hi) {
    const int64_t mid = lo + (hi - lo) / 2;
    if (P[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// log2 of the lanes per record for a task of R records and W items run by
// `warps` warps: batches small enough that every warp gets batches_per_warp
// of them, but no more lanes on a record than leave each lane_pairs pairs
// of 8 columns
__device__ __forceinline__ int32_t lanes_log2(int64_t R, int64_t W, int warps, const PlanParams &pp) {
  const int64_t per = R / (int64_t(pp.batches_per_warp) * warps);
  int lg_b = 0;
  while (lg_b < 5 && (int64_t(2) << lg_b) <= per) lg_b++;
  int lg_s = 5 - lg_b;
  const int64_t pairs = W / (8 * R) + 1;
  while (lg_s > 0 && (pairs >> lg_s) < pp.lane_pairs) lg_s--;
  return lg_s;
}

__device__ __forceinline__ Task make_task(int64_t v, int64_t k0, int64_t k1, int64_t r0, int64_t r1, int32_t lg_s) {
  Task t;
  t.k0 = k0;
  t.r0 = r0;
  t.v = int32_t(v);
  t.nrec = int32_t(k1 - k0);
  t.nmem = int32_t(r1 - r0);
  t.lg_s = lg_s;
  return t;
}

__global__ void k_plan_fill(int64_t nv, const int64_t *__restrict__ off, const int64_t *__restrict__ ioff,
                            const int64_t *__restrict__ P, const PlanParams pp, const int64_t *__restrict__ nb_pos,
                            const int64_t *__restrict__ nw_pos, const int64_t *__restrict__ nt_pos,
                            Task *__restrict__ bt, Task *__restrict__ wt, int32_t *__restrict__ tt) {
  XT_GRID_STRIDE(v, nv) {
    int64_t nb, nw, nt, parts, chunks, work;
    classify(v, off, ioff, P, pp, nb, nw, nt, parts, chunks, work);
    const int64_t k0 = ioff[v], k1 = ioff[v + 1];
    if (nt) tt[nt_pos[v]] = int32_t(v);
    if (nw) {
      // The lanes per record that take the warp the fewest steps. Records
      // are stored longest first, so a batch of 32 / S records runs as many
      // steps as its first record needs on S lanes (its pairs: the suffix
      // length plus an average offset into its first pair, over 8); each
      // batch also costs about one step of set-up.
      int32_t lg_s = 0;
      int64_t best = INT64_MAX;
      for (int32_t ls = 0; ls <= 5; ls++) {
        const int64_t B = int64_t(32) >> ls, S = int64_t(1) << ls;
        int64_t steps = 0;
        for (int64_t i = k0; i < k1; i += B) steps += 1 + ((P[i + 1] - P[i] + 11) / 8 + S - 1) / S;
        if (steps < best) {
          best = steps;
          lg_s = ls;
        }
      }
      wt[nw_pos[v]] = make_task(v, k0, k1, off[v], off[v + 1], lg_s);
    }
    if (!nb) continue;
    const int64_t base = P[k0];
    int64_t t = nb_pos[v], prev = k0;
    for (int64_t c = 0; c < chunks; c++) {
      const int64_t kend = (c + 1 == chunks) ? k1 : lower_bound_i64(P, prev, k1, base + (work * (c + 1)) / chunks);
      if (kend <= prev) continue;  // empty chunk (one in-record carries more work)
      // (a per-chunk step estimate like the warp tasks' bought 0.17 ms of
      // count at s24 for 5.8 ms of plan: one thread walks a head's chunks)
      const int32_t lg_s = lanes_log2(kend - prev, P[kend] - P[prev], kWarps, pp);
      for (int64_t p = 0; p < parts; p++) {
        const int64_t r0 = off[v] + p * kBlockDmax;
        const int64_t r1 = min(off[v + 1], r0 + kBlockDmax);
        bt[t++] = make_task(v, prev, kend, r0, r1, lg_s);
      }
      prev = kend;
    }
    for (; t < nb_pos[v] + nb; t++) bt[t] = make_task(v, k1, k1, off[v], off[v] + 1, 0);  // empty chunks: no-ops
  }
}

// CTA tasks run chunk-major: every head's first chunk, then every head's
// second, ... (key: chunk index within its head, then head). Tasks that run
// together then belong to many heads and read the same rows' suffixes while
// they are in L2 (R-MAT s24: 40.2 -> 38.6 ms against head-major order).
__global__ void k_task_keys(const Task *__restrict__ bt, int64_t n, const int64_t *__restrict__ nb_pos,
                            uint64_t *__restrict__ key, int32_t *__restrict__ idx) {
  XT_GRID_STRIDE(i, n) {
    const int64_t v = bt[i].v;
    key[i] = (uint64_t(i - nb_pos[v]) << 32) | uint64_t(v);
    idx[i] = int32_t(i);
  }
}

__global__ void k_task_gather(const Task *__restrict__ bt, const int32_t *__restrict__ idx, int64_t n,
                              Task *__restrict__ out) {
  XT_GRID_STRIDE(i, n) out[i] = bt[idx[i]];
}

// Global count, cluster tier: the cluster tasks of head v, for the heads
// whose CTA tasks would split N+(v) into parts (more than kBlockDmax
// members): parts of kClusterDmax members x chunks of kCluster * block_work
// items. Returns how many (0 for every other head).
__device__ __forceinline__ int64_t cluster_tasks(int64_t v, const int64_t *__restrict__ off,
                                                 const int64_t *__restrict__ ioff, const int64_t *__restrict__ P,
                                                 const PlanParams pp, int64_t &parts, int64_t &chunks,
                                                 int64_t &work) {
  int64_t nb, nw, nt, bparts, bchunks;
  classify(v, off, ioff, P, pp, nb, nw, nt, bparts, bchunks, work);
  parts = chunks = 0;
  if (nb == 0 || bparts <= 1) return 0;
  parts = (off[v + 1] - off[v] + kClusterDmax - 1) / kClusterDmax;
  const int64_t cw = pp.block_work * kCluster;
  chunks = (work + cw - 1) / cw;
  return parts * chunks;
}

__global__ void k_plan_ccount(int64_t nv, const int64_t *__restrict__ off, const int64_t *__restrict__ ioff,
                              const int64_t *__restrict__ P, const PlanParams pp, int64_t *__restrict__ nc_out) {
  XT_GRID_STRIDE(v, nv) {
    int64_t parts, chunks, work;
    nc_out[v] = cluster_tasks(v, off, ioff, P, pp, parts, chunks, work);
  }
}

__global__ void k_plan_cfill(int64_t nv, const int64_t *__restrict__ off, const int64_t *__restrict__ ioff,
                             const int64_t *__restrict__ P, const PlanParams pp, const int64_t *__restrict__ nc_pos,
                             Task *__restrict__ ct) {
  XT_GRID_STRIDE(v, nv) {
    int64_t parts, chunks, work;
    const int64_t n = cluster_tasks(v, off, ioff, P, pp, parts, chunks, work);
    if (!n) continue;
    const int64_t k0 = ioff[v], k1 = ioff[v + 1], base = P[k0];
    int64_t t = nc_pos[v], prev = k0;
    for (int64_t c = 0; c < chunks; c++) {
      const int64_t kend = (c + 1 == chunks) ? k1 : lower_bound_i64(P, prev, k1, base + (work * (c + 1)) / chunks);
      if (kend <= prev) continue;
      const int32_t lg_s = lanes_log2(kend - prev, P[kend] - P[prev], kWarps * kCluster, pp);
      for (int64_t p = 0; p < parts; p++) {
        const int64_t r0 = off[v] + p * kClusterDmax;
        const int64_t r1 = min(off[v + 1], r0 + kClusterDmax);
        ct[t++] = make_task(v, prev, kend, r0, r1, lg_s);
      }
      prev = kend;
    }
    for (; t < nc_pos[v] + n; t++) ct[t] = make_task(v, k1, k1, off[v], off[v] + 1, 0);  // empty chunks: no-ops
  }
}

// the CTA tasks of heads that are not cluster heads (at most kBlockDmax members)
struct NotClusterHead {
  const int64_t *off;
  __host__ __device__ bool operator()(const Task &t) const { return off[t.v + 1] - off[t.v] <= kBlockDmax; }
};

// ---- membership structures --------------------------------------------------

__device__ __forceinline__ uint32_t hash_slot(int32_t x, int shift) {
  return (uint32_t(x) * 0x9E3779B1u) >> shift;
}

// inserts x and returns its slot
__device__ __forceinline__ uint32_t hash_insert(int32_t *tab, uint32_t mask, int shift, int32_t x) {
  uint32_t h = hash_slot(x, shift);
  while (true) {
    const int32_t old = atomicCAS(&tab[h], kEmpty, x);
    if (old == kEmpty || old == x) return h;
    h = (h + 1) & mask;
  }
}

// Cuckoo table (global-count warp tasks): member x is stored as the key x + 1
// in one of its two slots h1, h2 (0 marks an empty slot, so an all-zero
// region is an empty table and an empty bitmap at once). Insertion follows
// Alcantara et al.'s parallel cuckoo hashing: swap the key into its slot,
// continue with the key it evicted at that key's other slot; a lane whose
// chain outlasts kCuckooIters reports failure and the task falls back to
// linear probing. A probe reads both slots, with no loop and no divergence.
constexpr uint32_t kCuckooMul1 = 0x9E3779B1u, kCuckooMul2 = 0x7FEB352Du;
constexpr int kCuckooIters = 64;  // eviction chain limit (a test hook can lower it)

__device__ __forceinline__ uint32_t cuckoo_h1(uint32_t key, int shift) { return (key * kCuckooMul1) >> shift; }
__device__ __forceinline__ uint32_t cuckoo_h2(uint32_t key, int shift) { return (key * kCuckooMul2) >> shift; }

__device__ __forceinline__ bool cuckoo_insert(int32_t *tab, int shift, uint32_t key, int iters) {
  uint32_t slot = cuckoo_h1(key, shift);
  for (int it = 0; it < iters; it++) {
    const uint32_t old = atomicExch(reinterpret_cast<unsigned int *>(&tab[slot]), key);
    if (old == 0u) return true;
    key = old;
    const uint32_t a = cuckoo_h1(key, shift);
    slot = (slot == a) ? cuckoo_h2(key, shift) : a;
  }
  return false;  // `key` is out of the table
}

// the slot holding x, or -1
__device__ __forceinline__ int hash_find(const int32_t *tab, uint32_t mask, int shift, int32_t x) {
  uint32_t h = hash_slot(x, shift);
  while (true) {
    const int32_t k = tab[h];
    if (k == x) return int(h);
    if (k == kEmpty) return -1;
    h = (h + 1) & mask;
  }
}

// The member set N+(v) (or one part of it) in shared memory.
struct Members {
  int32_t *words;   // bitmap words or hash slots
  uint16_t *idx;    // per-vertex and per-edge modes: per bitmap word, the index of its first
                    // member; per hash slot, the index of the member it holds
  int32_t *mcnt;    // same modes: per-member hit counters
  int32_t lo, hi;   // smallest and largest member
  uint32_t base;    // bitmap: x is bit (x & 31) of words[(x >> 5) - base]
  uint32_t nwords;  // bitmap: words in use; words[nwords] is a zero guard word
  uint32_t mask;    // hash: slots - 1
  int shift;        // hash: 32 - log2(slots)
  bool bitmap;
  bool cuckoo;      // hash kept as a cuckoo table (global-count warp tasks)
  uint32_t ctab;    // cluster tier: the shared-window address of the CTAs' tables
  int32_t cb[kCluster - 1];  // cluster tier: the first member of CTAs 1 .. kCluster-1
};

// Member-set kinds, one specialised streaming loop each.
constexpr int kKindHash = 0, kKindBitmap = 1, kKindCuckoo = 2, kKindCluster = 3;

// Chooses the structure for members mem[0, n) (ascending) that fits `words`
// words (a bitmap only while the members' id range is at most bitmap_bits)
// and returns how many words must be cleared. In the per-vertex and
// per-edge modes a bitmap also keeps, per word, the index of its first
// member, so a hit finds its member's counter by a popcount; a hash keeps
// the index of the member in each used slot.
template <bool PV>
__device__ __forceinline__ int members_layout(Members &m, const int32_t *mem, int n, int words, int64_t bitmap_bits) {
  m.lo = mem[0];
  m.hi = mem[n - 1];
  m.cuckoo = false;
  const int64_t range = int64_t(m.hi) - int64_t(m.lo) + 1;
  const int64_t nw = int64_t(m.hi >> 5) - int64_t(m.lo >> 5) + 1;
  m.bitmap = nw + 1 <= int64_t(words) && range <= bitmap_bits;
  if (m.bitmap) {
    m.base = uint32_t(m.lo >> 5);
    m.nwords = uint32_t(nw);
    m.mask = 0;
    m.shift = 0;
    return int(nw + 1);
  }
  m.base = m.nwords = 0;
  // every slot of the region (load factor <= 1/4, as n <= words / 4): the
  // emptier the table, the fewer lanes of a warp chase a probe chain, which
  // outweighs clearing the whole region per task (s24 31.75 -> 30.62 ms
  // against a table of 4n slots)
  int lg = 6;
  while ((2 << lg) <= words) lg++;
  m.mask = (1u << lg) - 1;
  m.shift = 32 - lg;
  return 1 << lg;
}

// inserts member i of mem[0, n) (ascending); with counters (per-vertex and
// per-edge modes) also records where the member's counter is found and
// clears it
template <bool PV>
__device__ __forceinline__ void members_insert_at(const Members &m, const int32_t *mem, int i) {
  const int32_t x = mem[i];
  if (m.bitmap) {
    const uint32_t wd = uint32_t(x >> 5) - m.base;
    atomicOr(reinterpret_cast<unsigned int *>(&m.words[wd]), 1u << (x & 31));
    if (PV && (i == 0 || uint32_t(mem[i - 1] >> 5) - m.base != wd)) m.idx[wd] = uint16_t(i);
  } else {
    const uint32_t slot = hash_insert(m.words, m.mask, m.shift, x);
    if (PV) m.idx[slot] = uint16_t(i);
  }
  if (PV) m.mcnt[i] = 0;
}

__device__ __forceinline__ void members_insert(const Members &m, int32_t x) {
  if (m.bitmap) {
    atomicOr(reinterpret_cast<unsigned int *>(&m.words[uint32_t(x >> 5) - m.base]), 1u << (x & 31));
  } else {
    hash_insert(m.words, m.mask, m.shift, x);
  }
}

// Global-count warp tasks: the member set in a warp slice that is all zero
// when the task starts: a bitmap over [min, max] when that fits, else a
// cuckoo table over every slot. Returns false (warp-uniform) when a cuckoo
// insert failed; the caller then rebuilds the set by linear probing.
__device__ __forceinline__ bool warp_set_build(Members &m, const int32_t *mem, int n, int words, int64_t bitmap_bits,
                                               int iters, int lane) {
  m.lo = mem[0];
  m.hi = mem[n - 1];
  const int64_t range = int64_t(m.hi) - int64_t(m.lo) + 1;
  const int64_t nw = int64_t(m.hi >> 5) - int64_t(m.lo >> 5) + 1;
  m.bitmap = nw + 1 <= int64_t(words) && range <= bitmap_bits;
  m.cuckoo = !m.bitmap;
  bool ok = true;
  if (m.bitmap) {
    m.base = uint32_t(m.lo >> 5);
    m.nwords = uint32_t(nw);
    m.mask = 0;
    m.shift = 0;
    for (int i = lane; i < n; i += 32) members_insert(m, mem[i]);
  } else {
    int lg = 6;
    while ((2 << lg) <= words) lg++;
    m.base = m.nwords = 0;
    m.mask = (1u << lg) - 1;
    m.shift = 32 - lg;
    for (int i = lane; i < n; i += 32) ok &= cuckoo_insert(m.words, m.shift, uint32_t(mem[i]) + 1u, iters);
  }
  return __all_sync(0xffffffffu, ok);
}

// Returns a warp slice to all zero: clears the bitmap words or cuckoo slots
// that members [0, n) took.
__device__ __forceinline__ void warp_set_reset(const Members &m, const int32_t *mem, int n, int lane) {
  for (int i = lane; i < n; i += 32) {
    const int32_t x = mem[i];
    if (m.bitmap) {
      m.words[uint32_t(x >> 5) - m.base] = 0;
    } else {
      const uint32_t key = uint32_t(x) + 1u, a = cuckoo_h1(key, m.shift);
      if (uint32_t(m.words[a]) == key) m.words[a] = 0;
      else m.words[cuckoo_h2(key, m.shift)] = 0;
    }
  }
}

__device__ __forceinline__ void zero_words(int32_t *w, int n, int t, int nt) {
  for (int i = 4 * t; i < n; i += 4 * nt) *reinterpret_cast<int4 *>(w + i) = make_int4(0, 0, 0, 0);
}

// ---- streaming the in-record suffixes ----------------------------------------
//
// A pair is an aligned 32-byte block of 8 columns (one 256-bit load) of the
// padded column array, where every row starts on a pair boundary and is
// padded with sentinels. A record's suffix covers pairs 0 .. np-1 of its
// row; the columns before the suffix in pair 0 are the row's own ids up to
// the head (below every member of N+(head)) and those after it in the last
// pair are sentinels, so no pair needs masking. A batch holds 32/S records;
// the S lanes of record j take its pairs k, k+S, ... Records of a head are
// stored longest first, so the lanes of a batch run for about as many steps.
constexpr int32_t kSentinel = kPadSentinel;  // negative: below every member, and not kEmpty
// positions inside one suffix are int32: out-degrees stay below this
constexpr int64_t kMaxOutDegree = kMaxRecLen;  // and the in-records' length field

// One 256-bit load per lane (sm_100 vector width; the column array is
// 256-byte aligned, so every pair is 32-byte aligned): one L1 wavefront per
// line touched instead of one per 16-byte half. A record's lanes walk
// consecutive pairs, so each load asks L2 for the 256 bytes around it (the
// next steps' pairs) and skips L1, where a pair is never read twice (s22
// 5.74 -> 5.62 ms, s24 32.02 -> 31.77 ms).
// Pair indices fit 32 bits (the padded columns number below 2^35): a lane
// steps its pair index and forms the address with 32-bit arithmetic
#ifndef XT_P32
#define XT_P32 1
#endif
#if XT_P32
using PairIdx = uint32_t;
#else
using PairIdx = int64_t;
#endif
__device__ __forceinline__ void load_pair(const int32_t *__restrict__ col, PairIdx P, int4 &a, int4 &b) {
  const int32_t *p = col + (uint64_t(P) << 3);
  asm volatile("ld.global.nc.L1::no_allocate.L2::256B.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(a.x), "=r"(a.y), "=r"(a.z), "=r"(a.w), "=r"(b.x), "=r"(b.y), "=r"(b.z), "=r"(b.w)
               : "l"(p));
}

// Asks L2 to fetch [p, p + bytes) (16-byte aligned, a multiple of 16 bytes)
// without waiting for it.
__device__ __forceinline__ void prefetch_l2(const void *p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Asks L2 for the line holding p (no register result, nothing to wait for).
__device__ __forceinline__ void prefetch_line_l2(const void *p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// bitmap membership: bit (w & 31) of word (w >> 5) - base; every w outside
// the bitmap's words lands on the zero guard word
__device__ __forceinline__ uint32_t bitmap_test(const Members &m, int32_t w) {
  uint32_t i = uint32_t(w >> 5) - m.base;
  i = i < m.nwords ? i : m.nwords;
  const uint32_t x = uint32_t(m.words[i]);
  return __funnelshift_r(x, x, uint32_t(w)) & 1u;
}

template <bool PV>
__device__ __forceinline__ int hash_test(const Members &m, int32_t w) {
  if (uint32_t(w - m.lo) > uint32_t(m.hi - m.lo)) return 0;  // sentinels too
  const int slot = hash_find(m.words, m.mask, m.shift, w);
  if (slot < 0) return 0;
  if (PV) atomicAdd(&m.mcnt[m.idx[slot]], 1);
  return 1;
}

// cuckoo membership: the key w + 1 in either of its two slots (sentinels and
// ids outside the set match no stored key)
__device__ __forceinline__ uint32_t cuckoo_test(const Members &m, int32_t w) {
  const uint32_t key = uint32_t(w) + 1u;
  const uint32_t x = uint32_t(m.words[cuckoo_h1(key, m.shift)]);
  const uint32_t y = uint32_t(m.words[cuckoo_h2(key, m.shift)]);
  return uint32_t(x == key) | uint32_t(y == key);
}

// the shared::cluster address of the same shared-memory offset in CTA
// `rank` of this cluster
__device__ __forceinline__ uint32_t cluster_addr(uint32_t local, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local), "r"(rank));
  return r;
}
__device__ __forceinline__ int32_t ld_cluster(uint32_t addr) {
  int32_t v;
  asm volatile("ld.shared::cluster.s32 %0, [%1];" : "=r"(v) : "r"(addr));
  return v;
}

// cluster membership: CTA c of the cluster holds the members from cb[c-1]
// up to cb[c] in a linear-probing table (at most kBlockDmax members in
// kBlockWords slots, so every probe chain ends at an empty slot); w is
// looked up in the table of the CTA whose range holds it
__device__ __forceinline__ uint32_t cluster_test(const Members &m, int32_t w) {
  if (uint32_t(w - m.lo) > uint32_t(m.hi - m.lo)) return 0u;  // sentinels too
  uint32_t owner = 0;
#pragma unroll
  for (int c = 0; c < kCluster - 1; c++) owner += uint32_t(w >= m.cb[c]);
  const uint32_t base = cluster_addr(m.ctab, owner);
  uint32_t h = hash_slot(w, m.shift);
  while (true) {
    const int32_t k = ld_cluster(base + 4u * h);
    if (k == w) return 1u;
    if (k == kEmpty) return 0u;
    h = (h + 1) & m.mask;
  }
}

template <bool PV, int KIND>
__device__ __forceinline__ int probe_pair(const int4 a, const int4 b, const Members &m) {
  if (KIND == kKindCluster) {
    return int((cluster_test(m, a.x) + cluster_test(m, a.y)) + (cluster_test(m, a.z) + cluster_test(m, a.w)) +
               (cluster_test(m, b.x) + cluster_test(m, b.y)) + (cluster_test(m, b.z) + cluster_test(m, b.w)));
  }
  if (KIND == kKindBitmap) {
    return int((bitmap_test(m, a.x) + bitmap_test(m, a.y)) + (bitmap_test(m, a.z) + bitmap_test(m, a.w)) +
               (bitmap_test(m, b.x) + bitmap_test(m, b.y)) + (bitmap_test(m, b.z) + bitmap_test(m, b.w)));
  }
  if (KIND == kKindCuckoo) {
    return int((cuckoo_test(m, a.x) + cuckoo_test(m, a.y)) + (cuckoo_test(m, a.z) + cuckoo_test(m, a.w)) +
               (cuckoo_test(m, b.x) + cuckoo_test(m, b.y)) + (cuckoo_test(m, b.z) + cuckoo_test(m, b.w)));
  }
  return hash_test<PV>(m, a.x) + hash_test<PV>(m, a.y) + hash_test<PV>(m, a.z) + hash_test<PV>(m, a.w) +
         hash_test<PV>(m, b.x) + hash_test<PV>(m, b.y) + hash_test<PV>(m, b.z) + hash_test<PV>(m, b.w);
}

// Per-vertex and per-edge modes: a hit bumps its member's counter (bitmap:
// the member's index is the word's first index plus the set bits below;
// hash: the index kept beside its slot) and, per edge, the edge u->w at
// column position pos
// the shared-window address of a shared-memory pointer
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// atomic add of 1 to a shared counter when pred != 0: the instruction is
// predicated, so lanes that do not add take no branch (the address may be
// garbage when pred == 0; it is not accessed)
__device__ __forceinline__ void red_shared_add1_if(uint32_t saddr, uint32_t pred) {
  asm volatile("{\n .reg .pred q;\n setp.ne.u32 q, %1, 0;\n @q red.shared.add.u32 [%0], 1;\n}" ::"r"(saddr),
               "r"(pred)
               : "memory");
}

template <int MODE, int KIND>
__device__ __forceinline__ int probe_one(const Members &m, int32_t w, unsigned int *__restrict__ es, int64_t pos) {
  if (XT_PV_PRED && MODE == 1 && KIND == kKindBitmap) {
    // per-vertex mode, branch-free: every candidate finds the counter its
    // member would have (the word's first member index plus the set bits
    // below; idx of a word without members, or of the guard word, is stale
    // and then unused) and the increment is predicated on the hit. R-MAT s24
    // 63.8 -> 60.4 ms; the per-edge mode keeps its branch (its predicated
    // global increments measured 97.0 -> 98.8 ms, and its member counter
    // alone predicated 94.0 -> 95.5 ms)
    uint32_t i = uint32_t(w >> 5) - m.base;
    i = i < m.nwords ? i : m.nwords;
    const uint32_t x = uint32_t(m.words[i]);
    const uint32_t bit = uint32_t(w) & 31u;
    const uint32_t hit = (x >> bit) & 1u;
    const uint32_t k = uint32_t(m.idx[i]) + uint32_t(__popc(x & ((1u << bit) - 1u)));
    red_shared_add1_if(smem_u32(m.mcnt) + 4u * k, hit);
    return int(hit);
  }
  if (KIND == kKindBitmap) {
    uint32_t i = uint32_t(w >> 5) - m.base;
    i = i < m.nwords ? i : m.nwords;
    const uint32_t x = uint32_t(m.words[i]);
    const uint32_t bit = uint32_t(w) & 31u;
    if (!((x >> bit) & 1u)) return 0;  // the guard word is zero: i < nwords below
    atomicAdd(&m.mcnt[m.idx[i] + __popc(x & ((1u << bit) - 1u))], 1);
  } else if (!hash_test<true>(m, w)) {
    return 0;
  }
  if (MODE == 2) atomicAdd(&es[pos], 1u);
  return 1;
}

template <int MODE, int KIND>
__device__ __forceinline__ int probe_pair_counted(const int4 a, const int4 b, const Members &m,
                                                  unsigned int *__restrict__ es, int64_t pos0) {
  return probe_one<MODE, KIND>(m, a.x, es, pos0) + probe_one<MODE, KIND>(m, a.y, es, pos0 + 1) +
         probe_one<MODE, KIND>(m, a.z, es, pos0 + 2) + probe_one<MODE, KIND>(m, a.w, es, pos0 + 3) +
         probe_one<MODE, KIND>(m, b.x, es, pos0 + 4) + probe_one<MODE, KIND>(m, b.y, es, pos0 + 5) +
         probe_one<MODE, KIND>(m, b.z, es, pos0 + 6) + probe_one<MODE, KIND>(m, b.w, es, pos0 + 7);
}

// Streams the suffixes of in-records [k0, kend) through the member set with
// 2^lg_s lanes per record, in batches claimed from `cursor` (shared by the
// warps of a CTA task) or taken in order (cursor null); returns this lane's
// hits. Per-vertex mode (MODE 1) credits each record's hits to its owner u;
// per-edge mode (MODE 2) credits them to the record's own edge u->v and each
// hit to the edge u->w at the candidate's column, both at padded column
// positions (no per-record load of the tail or its row offsets).
// PF: a bulk L2 prefetch of each record's suffix one batch ahead (one per
// record, by the record's first lane): it pays where little of the graph is
// re-read from L2 (the 4,096-graph batch: 40.3 -> 34.6 ms) and costs issue
// slots where much is (R-MAT s24: 28.55 -> 30.4 ms), so it is chosen per
// graph (xt_graph_set_prefetch, the autotuner)
template <int MODE, int KIND, bool PF>
__device__ __forceinline__ int64_t stream_kind(const InRec *__restrict__ rec, const int32_t *__restrict__ rec_u,
                                               const int32_t *__restrict__ colp, int64_t k0, int64_t kend, int lg_s,
                                               int *cursor, const Members &m,
                                               int64_t *__restrict__ pv, unsigned int *__restrict__ es,
                                               const int64_t *__restrict__ off, const int64_t *__restrict__ poff,
                                               int lane, int bstride = 1, int boff = 0) {
  constexpr bool PV = MODE != 0;
  const int S = 1 << lg_s;
  const int bsz = 32 >> lg_s;
  const int j = lane >> lg_s, k = lane & (S - 1);
  const int32_t nrec = int32_t(kend - k0);
  const int4 sent = make_int4(kSentinel, kSentinel, kSentinel, kSentinel);
  rec += k0;
  if (MODE == 1) rec_u += k0;
  int32_t seq = 0;
  auto claim = [&]() -> int32_t {
    if (!cursor) {
      const int32_t b = seq;
      seq += bsz;
      return b;
    }
    int c = 0;
    if (lane == 0) c = atomicAdd(cursor, bsz);
    // batch c / bsz of this caller is batch (c / bsz) * bstride + boff of the
    // task (a cluster's CTAs take every kCluster-th batch each)
    return __shfl_sync(0xffffffffu, c, 0) * bstride + boff * bsz;
  };
  // a record as {pair, lw, 0, u} (u only in the per-vertex mode)
  auto fetch = [&](int32_t base) -> int4 {
    const int32_t r = base + j;
    const uint2 x = r < nrec ? __ldg(reinterpret_cast<const uint2 *>(rec) + r) : make_uint2(0u, 0u);
    return make_int4(int(x.x), int(x.y), 0, (MODE == 1 && r < nrec) ? __ldg(rec_u + r) : -1);
  };
  // records are loaded two batches ahead (an L2 prefetch of the next batch's
  // suffixes cost more instructions than the latency it hid: s24 38.5 ms
  // with it, 36.2 ms without)
  int32_t kb = claim();
  int4 r4 = fetch(kb);
  int32_t nkb = claim();
  int4 n4 = fetch(nkb);
  int64_t hits = 0;
  while (kb < nrec) {  // warp-uniform
    const int32_t nnkb = claim();
    const int4 nn4 = fetch(nnkb);
    const int32_t nlen = int32_t(uint32_t(n4.y) & uint32_t(kMaxRecLen - 1));
    if (PF && k == 0 && nlen > 0) {
      // the next batch's suffix into L2 while this batch streams (its record
      // arrived a batch ago): one bulk prefetch per record, at most 64 KB
      const int64_t nb = int64_t((int32_t(uint32_t(n4.y) >> kRecLenBits) + nlen + 7) >> 3) * 32;
      prefetch_l2(colp + (int64_t(uint32_t(n4.x)) << 3), uint32_t(nb < 65536 ? nb : 65536));
    }
    const int64_t s = (int64_t(uint32_t(r4.x)) << 3) | int64_t(uint32_t(r4.y) >> kRecLenBits);
    const int32_t len = int32_t(uint32_t(r4.y) & uint32_t(kMaxRecLen - 1));
    const int32_t np = len > 0 ? (int32_t(s & 7) + len + 7) >> 3 : 0;  // pairs of the suffix
    const int32_t cnt = np > k ? ((np - k + S - 1) >> lg_s) : 0;            // this lane's
    const int32_t steps = int32_t(__reduce_max_sync(0xffffffffu, uint32_t(cnt)));
    PairIdx P = PairIdx(uint32_t(r4.x)) + PairIdx(k);  // r4.x = s >> 3
    int4 xa = sent, xb = sent;
    if (cnt > 0) load_pair(colp, P, xa, xb);
    int h = 0;
#if XT_LANE_LOOP
    // each lane runs its own pairs and leaves the loop after its last one
    for (int32_t it = 0; it < cnt; it++) {
      const int4 a = xa, b = xb;
      const PairIdx pa = P;  // the pair in a, b
      P += S;
      if (it + 1 < cnt) load_pair(colp, P, xa, xb);  // next step's pair in flight during the probes
      if (PV) h += probe_pair_counted<MODE, KIND>(a, b, m, es, 8 * int64_t(pa));
      else h += probe_pair<false, KIND>(a, b, m);
    }
    (void)steps;
#else
    // a lane past its last pair probes sentinels
    for (int32_t it = 0; it < steps; it++) {
      const int4 a = xa, b = xb;
      const PairIdx pa = P;  // the pair in a, b
      P += S;
      if (it + 1 < cnt) {
        load_pair(colp, P, xa, xb);  // next step's pair in flight during the probes
#if XT_PF_DIST > 1
        if (it + XT_PF_DIST < cnt) prefetch_line_l2(colp + 8 * (int64_t(P) + int64_t(XT_PF_DIST - 1) * S));
#endif
      } else {
        xa = sent;
        xb = sent;
      }
      if (PV) h += probe_pair_counted<MODE, KIND>(a, b, m, es, 8 * int64_t(pa));
      else h += probe_pair<false, KIND>(a, b, m);
    }
#endif
    if (PV) {
      int hr = h;
#pragma unroll
      for (int o = 16; o; o >>= 1)
        if (o < S) hr += __shfl_down_sync(0xffffffffu, hr, o, S);
      if (MODE == 1 && k == 0 && hr && r4.w >= 0)
        atomicAdd(reinterpret_cast<unsigned long long *>(&pv[r4.w]), (unsigned long long)hr);
      if (MODE == 2 && k == 0 && hr) atomicAdd(&es[s - 1], unsigned(hr));  // the edge u->v
    }
    hits += h;
    kb = nkb;
    r4 = n4;
    nkb = nnkb;
    n4 = nn4;
  }
  return hits;
}

template <int MODE, bool PF>
__device__ __forceinline__ int64_t stream_suffixes(const InRec *__restrict__ rec, const int32_t *__restrict__ rec_u,
                                                   const int32_t *__restrict__ colp, int64_t k0, int64_t kend,
                                                   int lg_s, int *cursor, const Members &m,
                                                   int64_t *__restrict__ pv, unsigned int *__restrict__ es,
                                                   const int64_t *__restrict__ off, const int64_t *__restrict__ poff,
                                                   int lane) {
  // the membership kind is fixed per task: one specialised loop each
  if (m.bitmap)
    return stream_kind<MODE, kKindBitmap, PF>(rec, rec_u, colp, k0, kend, lg_s, cursor, m, pv, es, off, poff, lane);
  if (MODE == 0 && kWarpCuckoo && m.cuckoo)
    return stream_kind<MODE, kKindCuckoo, PF>(rec, rec_u, colp, k0, kend, lg_s, cursor, m, pv, es, off, poff, lane);
  return stream_kind<MODE, kKindHash, PF>(rec, rec_u, colp, k0, kend, lg_s, cursor, m, pv, es, off, poff, lane);
}

// ---- the count kernel ---------------------------------------------------------

struct CountArgs {
  const int64_t *off;
  const int32_t *col;
  const int32_t *colp;  // padded columns (suffixes are streamed from here)
  const int64_t *poff;  // padded row starts
  const int64_t *ioff;
  const InRec *rec;
  const int32_t *rec_u;  // the records' tails (per-vertex and per-edge modes)
  const Task *bt;  // CTA tasks
  int64_t n_bt;
  const Task *wt;  // warp tasks
  int64_t n_wt;
  const int32_t *tt;  // lane tasks (heads)
  int64_t n_tt;
  const Task *ct;  // cluster tasks
  int64_t n_ct;
  int lane_merge;  // lane tasks: members found by a two-pointer merge (1) or binary search (0)
  int64_t stride;  // task lists hold every stride-th task of the schedule (a shard of it), else 1
  int claim;       // warp tasks (and groups of 32 lane tasks) taken from their cursor per atomic
  unsigned long long *cursor;     // [0] CTA, [1] warp, [2] lane task cursors
  unsigned long long *global;     // the total
  int64_t *pv;                    // per-vertex counts (per-vertex mode)
  unsigned int *es;               // per-edge counts, out-CSR order (per-edge mode)
  const int32_t *group;           // head -> group (a graph of a batch), or null
  unsigned long long *group_out;  // per-group counts when group != null
  int64_t bitmap_bits;            // largest member id range kept as a bitmap
  int cuckoo_iters;               // cuckoo eviction chain limit
  int *err;                       // error word: kErrStageTimeout when a staging wait gave up
};

// adds a warp's hits of one task to the task head's group
__device__ __forceinline__ void credit_group(const CountArgs &a, int64_t v, int64_t h, int lane) {
  for (int o = 16; o; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
  if (lane == 0 && h) atomicAdd(&a.group_out[a.group[v]], (unsigned long long)h);
}

__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gsrc) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// CTA-task staging by one bulk copy (global -> this CTA's shared memory, no
// multicast) completed on an mbarrier that counts its bytes.
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// waits for phase `parity` of the barrier, at most kStageWaitLimit tries
constexpr uint32_t kStageWaitLimit = 1u << 22;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
  for (uint32_t it = 0; it < kStageWaitLimit; it++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// the generic-proxy reads of the staging buffer are ordered before the next
// bulk copy (async proxy) overwrites it
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Task staging: the next task's descriptor is claimed and its members copied
// into shared memory (cp.async) and its in-records sent to L2 while the
// current task streams, so a task starts without a round trip to memory.
constexpr int kStageCta = kBlockDmax + 8;   // members, from r0 rounded down to 4 columns
constexpr int kStageWarp = kWarpDmax + 8;
constexpr int kStageInts = (kStageCta > kWarps * kStageWarp) ? kStageCta : kWarps * kStageWarp;

// the next task from `cursor` (warp-uniform); nrec = -1 when none is left.
// A shard's list is every stride-th task of the schedule's (tasks points at
// its first, n counts its own).
__device__ __forceinline__ Task claim_task(unsigned long long *cursor, const Task *__restrict__ tasks, int64_t n,
                                           int64_t stride, int lane) {
  unsigned long long i = 0;
  if (lane == 0) i = atomicAdd(cursor, 1ull);
  i = __shfl_sync(0xffffffffu, i, 0);
  if (int64_t(i) >= n) {
    Task t;
    t.k0 = t.r0 = 0;
    t.v = t.nmem = t.lg_s = 0;
    t.nrec = -1;
    return t;
  }
  return tasks[int64_t(i) * stride];
}

// Warp tasks (and lane tasks, 32 heads a group) are claimed from their
// global cursor `claim` at a time (lane 0 keeps the block), so the warps of
// the whole GPU take one atomic on that one address per `claim` tasks. Where
// tasks are many and small (the 4,096-graph batch: 38.2 -> 30.4 ms with 4)
// that atomic is the limit; elsewhere a block lengthens the tail (R-MAT s22
// 4.69 -> 4.79 ms with 4; s24 and Chung-Lu unchanged), so a plain graph
// claims one at a time and a batch four (xt_graph_set_claim, the autotuner).
struct ClaimBlock {
  unsigned long long next = 0, end = 0;  // lane 0: the unclaimed rest of its block
};
__device__ __forceinline__ Task claim_task_block(ClaimBlock &cb, unsigned long long *cursor,
                                                 const Task *__restrict__ tasks, int64_t n, int64_t stride, int claim,
                                                 int lane) {
  unsigned long long i = 0;
  if (lane == 0) {
    if (cb.next == cb.end) {
      cb.next = atomicAdd(cursor, (unsigned long long)claim);
      cb.end = cb.next + claim;
    }
    i = cb.next++;
  }
  i = __shfl_sync(0xffffffffu, i, 0);
  if (int64_t(i) >= n) {
    Task t;
    t.k0 = t.r0 = 0;
    t.v = t.nmem = t.lg_s = 0;
    t.nrec = -1;
    return t;
  }
  return tasks[int64_t(i) * stride];
}

// one warp: the task's records to L2, from the 16-byte boundary at or below
// the first (a record is 8 bytes; the record array's 16 bytes of slack keep
// the rounded-up end inside it), in pieces of at most 64 KB
__device__ __forceinline__ void prefetch_records(const InRec *__restrict__ rec, const Task &t, int lane) {
  const uintptr_t p0 = reinterpret_cast<uintptr_t>(rec + t.k0), a0 = p0 & ~uintptr_t(15);
  const int64_t bytes = int64_t((p0 + uintptr_t(t.nrec) * sizeof(InRec) - a0 + 15) & ~uintptr_t(15));
  for (int64_t q = int64_t(lane) << 16; q < bytes; q += int64_t(32) << 16)
    prefetch_l2(reinterpret_cast<const char *>(a0) + q, uint32_t(bytes - q < 65536 ? bytes - q : 65536));
}

// one warp: copies the task's members into stage and prefetches its records
// to L2; returns where the members start in stage
__device__ __forceinline__ int stage_task(int32_t *stage, const int32_t *__restrict__ col,
                                          const InRec *__restrict__ rec, const Task &t, int lane) {
  if (t.nrec < 0) return 0;
  const int64_t a0 = t.r0 & ~int64_t(3);
  const int nchunk = int((t.r0 + t.nmem - a0 + 3) >> 2);  // reads stay inside the column padding
  for (int i = lane; i < nchunk; i += 32) cp_async16(stage + 4 * i, col + a0 + 4 * i);
  cp_async_commit();
  prefetch_records(rec, t, lane);
  return int(t.r0 - a0);
}

// CTA tasks: one lane copies the task's members into stage with one bulk
// copy on the barrier (a plain arrival when there is no task, so the phase
// still completes), and warp 0's lanes send its in-records to L2; returns
// where the members start in stage
__device__ __forceinline__ int stage_task_bulk(int32_t *stage, uint64_t *bar, const int32_t *__restrict__ col,
                                               const InRec *__restrict__ rec, const Task &t, int lane) {
  if (lane == 0) {
    if (t.nrec < 0) {
      mbar_arrive(bar);
    } else {
      // from r0 rounded down to 4 columns (the column array is 256-byte
      // aligned), whole 16-byte chunks: reads stay inside the column padding
      const int64_t a0 = t.r0 & ~int64_t(3);
      const uint32_t bytes = uint32_t((t.r0 + t.nmem - a0 + 3) >> 2) * 16u;
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(bar, bytes);
      bulk_copy_g2s(stage, col + a0, bytes, bar);
    }
  }
  if (t.nrec < 0) return 0;
  prefetch_records(rec, t, lane);
  return int(t.r0 & 3);
}

// clears the first nclear words of the member set (thread t of nt)
template <bool PV>
__device__ __forceinline__ void clear_members(const Members &m, int nclear, int t, int nt) {
  for (int i = t; i < nclear; i += nt) m.words[i] = m.bitmap ? 0 : kEmpty;
}

// MODE 0: global count; 1: and per-vertex counts; 2: and per-edge counts.
// PF: bulk suffix prefetch (see stream_kind).
template <int MODE, bool PF>
// (the per-vertex and per-edge modes hold 56 KB of shared memory, so three
// of their CTAs fit an SM: their register budget is sized for three)
__global__ void __launch_bounds__(kThreads, MODE == 0 ? kMinBlocks : 3) k_count(const CountArgs a) {
  const int64_t *__restrict__ off = a.off;
  const int32_t *__restrict__ col = a.col;
  const int64_t *__restrict__ ioff = a.ioff;
  const InRec *__restrict__ rec = a.rec;
  unsigned long long *__restrict__ cursor = a.cursor;
  constexpr bool PV = MODE != 0;  // member sets with per-member hit counters
  int64_t *__restrict__ pv = a.pv;
  unsigned int *__restrict__ es = a.es;
  extern __shared__ int32_t smem[];
  int32_t *bwords = smem;  // kBlockWords
  // modes 1, 2: kBlockWords 16-bit member indices (bitmap word starts or
  // hash slot owners), then kBlockDmax member counters
  uint16_t *bidx = reinterpret_cast<uint16_t *>(smem + kBlockWords);
  int32_t *bmcnt = smem + kBlockWords + kBlockWords / 2;
  __shared__ __align__(16) int32_t s_stage[kStageInts];
  __shared__ __align__(8) uint64_t s_stage_bar;  // completes when a CTA task's members have landed
  __shared__ Task s_task[2];
  __shared__ int s_soff[2];
  __shared__ int s_batch;  // next in-record batch of the current CTA task
  __shared__ unsigned long long s_red[kWarps];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int64_t acc = 0;

  // ---- CTA tasks ----
  if (tid == 0) mbar_init(&s_stage_bar, 1);
  __syncthreads();
  uint32_t stage_parity = 0;
  if (warp == 0) {
    const Task t0 = claim_task(&cursor[0], a.bt, a.n_bt, a.stride, lane);
    const int so = stage_task_bulk(s_stage, &s_stage_bar, col, rec, t0, lane);
    if (lane == 0) {
      s_task[0] = t0;
      s_soff[0] = so;
    }
  }
  for (int cur = 0;; cur ^= 1) {
    // every thread waits for the staged members (bounded: on a timeout the
    // CTA leaves its task loop and reports it through the error word)
    const bool landed = mbar_wait_bounded(&s_stage_bar, stage_parity);
    stage_parity ^= 1u;
    if (tid == 0) s_batch = 0;
    if (__syncthreads_or(!landed)) {
      if (tid == 0 && a.err) atomicOr(a.err, kErrStageTimeout);
      break;
    }
    const Task t = s_task[cur];
    if (t.nrec < 0) break;
    const int32_t *mem = s_stage + s_soff[cur];
    Members m;
    m.words = bwords;
    m.idx = bidx;
    m.mcnt = bmcnt;
    const int nclear = members_layout<PV>(m, mem, t.nmem, kBlockWords, a.bitmap_bits);
    if (MODE == 0 && kWarpCuckoo && !m.bitmap) {
      // a hashed set as a cuckoo table over every slot (load <= 1/4); if a
      // chain runs too long anywhere, the task falls back to linear probing
      m.cuckoo = true;
      zero_words(bwords, nclear, tid, kThreads);
      __syncthreads();
      bool ok = true;
      for (int i = tid; i < t.nmem; i += kThreads)
        ok &= cuckoo_insert(m.words, m.shift, uint32_t(mem[i]) + 1u, a.cuckoo_iters);
      if (__syncthreads_or(!ok)) {
        m.cuckoo = false;
        clear_members<PV>(m, nclear, tid, kThreads);
        __syncthreads();
        for (int i = tid; i < t.nmem; i += kThreads) members_insert_at<PV>(m, mem, i);
        __syncthreads();
      }
    } else {
      clear_members<PV>(m, nclear, tid, kThreads);
      __syncthreads();
      for (int i = tid; i < t.nmem; i += kThreads) members_insert_at<PV>(m, mem, i);
      __syncthreads();
    }
    if (warp == 0) {  // stage is free again: bring in the next task
      const Task tn = claim_task(&cursor[0], a.bt, a.n_bt, a.stride, lane);
      const int so = stage_task_bulk(s_stage, &s_stage_bar, col, rec, tn, lane);
      if (lane == 0) {
        s_task[cur ^ 1] = tn;
        s_soff[cur ^ 1] = so;
      }
    }
    int64_t h = stream_suffixes<MODE, PF>(rec, a.rec_u, a.colp, t.k0, t.k0 + t.nrec, t.lg_s, &s_batch, m, pv, es, off, a.poff,
                                      lane);
    acc += h;
    if (a.group) credit_group(a, t.v, h, lane);
    if (PV) {
      for (int o = 16; o; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
      if (lane == 0) s_red[warp] = (unsigned long long)h;
    }
    __syncthreads();
    if (MODE == 1) {
      if (tid == 0) {
        unsigned long long tot = 0;
        for (int w = 0; w < kWarps; w++) tot += s_red[w];
        if (tot) atomicAdd(reinterpret_cast<unsigned long long *>(&pv[t.v]), tot);
      }
      for (int i = tid; i < t.nmem; i += kThreads)
        if (bmcnt[i]) atomicAdd(reinterpret_cast<unsigned long long *>(&pv[col[t.r0 + i]]), (unsigned long long)bmcnt[i]);
    }
    if (MODE == 2) {  // the counts sit at padded positions: this part's start in row v
      const int64_t pr0 = a.poff[t.v] + (t.r0 - off[t.v]);
      for (int i = tid; i < t.nmem; i += kThreads)
        if (bmcnt[i]) atomicAdd(&es[pr0 + i], unsigned(bmcnt[i]));
    }
    if (PV) __syncthreads();
  }

  // ---- warp tasks: the CTA region split among the warps ----
  ClaimBlock wclaim;
  if (MODE == 0 && kWarpCuckoo) {
    // The slice holds the CTA tasks' last set: zero it once. A task then
    // builds its bitmap or cuckoo table into the zeroed slice and, when done,
    // clears only the words or slots its members took, instead of clearing
    // the whole 1,024-word slice per task.
    int32_t *wstage = s_stage + warp * kStageWarp;
    int32_t *words = bwords + warp * kWarpWords;
    Task t = claim_task_block(wclaim, &cursor[1], a.wt, a.n_wt, a.stride, a.claim, lane);
    int so = stage_task(wstage, col, rec, t, lane);
    zero_words(words, kWarpWords, lane, 32);
    while (true) {
      cp_async_wait_all();
      __syncwarp();
      if (t.nrec < 0) break;
      const int32_t *mem = wstage + so;
      Members m;
      m.words = words;
      m.idx = nullptr;
      m.mcnt = nullptr;
      const bool ok = warp_set_build(m, mem, t.nmem, kWarpWords, a.bitmap_bits, a.cuckoo_iters, lane);
      __syncwarp();
      const Task tn = claim_task_block(wclaim, &cursor[1], a.wt, a.n_wt, a.stride, a.claim, lane);  // read after the stream
      int64_t h;
      if (ok) {
        h = stream_suffixes<MODE, PF>(rec, a.rec_u, a.colp, t.k0, t.k0 + t.nrec, t.lg_s, nullptr, m, pv, es, off, a.poff, lane);
        __syncwarp();
        warp_set_reset(m, mem, t.nmem, lane);
      } else {
        // a cuckoo chain ran too long (rare): the same members by linear
        // probing over the whole slice, which is zeroed again afterwards
        zero_words(words, kWarpWords, lane, 32);
        __syncwarp();
        const int nclear = members_layout<false>(m, mem, t.nmem, kWarpWords, a.bitmap_bits);
        clear_members<false>(m, nclear, lane, 32);
        __syncwarp();
        for (int i = lane; i < t.nmem; i += 32) members_insert_at<false>(m, mem, i);
        __syncwarp();
        h = stream_suffixes<MODE, PF>(rec, a.rec_u, a.colp, t.k0, t.k0 + t.nrec, t.lg_s, nullptr, m, pv, es, off, a.poff, lane);
        __syncwarp();
        zero_words(words, kWarpWords, lane, 32);
      }
      acc += h;
      if (a.group) credit_group(a, t.v, h, lane);
      __syncwarp();
      so = stage_task(wstage, col, rec, tn, lane);
      t = tn;
    }
  } else {
    int32_t *wstage = s_stage + warp * kStageWarp;
    Task t = claim_task_block(wclaim, &cursor[1], a.wt, a.n_wt, a.stride, a.claim, lane);
    int so = stage_task(wstage, col, rec, t, lane);
    while (true) {
      cp_async_wait_all();
      __syncwarp();
      if (t.nrec < 0) break;
      const int32_t *mem = wstage + so;
      Members m;
      m.words = bwords + warp * kWarpWords;
      m.idx = bidx + warp * kWarpWords;
      m.mcnt = bmcnt + warp * kWarpDmax;
      const int nclear = members_layout<PV>(m, mem, t.nmem, kWarpWords, a.bitmap_bits);
      clear_members<PV>(m, nclear, lane, 32);
      __syncwarp();
      for (int i = lane; i < t.nmem; i += 32) members_insert_at<PV>(m, mem, i);
      __syncwarp();
      const Task tn = claim_task_block(wclaim, &cursor[1], a.wt, a.n_wt, a.stride, a.claim, lane);  // read after the stream
      int64_t h = stream_suffixes<MODE, PF>(rec, a.rec_u, a.colp, t.k0, t.k0 + t.nrec, t.lg_s, nullptr, m, pv, es, off, a.poff,
                                        lane);
      acc += h;
      if (a.group) credit_group(a, t.v, h, lane);
      if (MODE == 1) {
        for (int o = 16; o; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
        __syncwarp();
        if (lane == 0 && h) atomicAdd(reinterpret_cast<unsigned long long *>(&pv[t.v]), (unsigned long long)h);
        for (int i = lane; i < t.nmem; i += 32)
          if (m.mcnt[i])
            atomicAdd(reinterpret_cast<unsigned long long *>(&pv[mem[i]]), (unsigned long long)m.mcnt[i]);
      }
      if (MODE == 2) {
        __syncwarp();
        const int64_t pr0 = a.poff[t.v] + (t.r0 - off[t.v]);
        for (int i = lane; i < t.nmem; i += 32)
          if (m.mcnt[i]) atomicAdd(&es[pr0 + i], unsigned(m.mcnt[i]));
      }
      __syncwarp();
      so = stage_task(wstage, col, rec, tn, lane);
      t = tn;
    }
  }

  // ---- lane tasks: one small head per lane ----
  // Each candidate w of a record's suffix is found in N+(v) (ascending) from
  // the position after the previous one: by binary search (MERGE = false),
  // or by stepping forward, a two-pointer merge of the suffix with N+(v)
  // (MERGE = true; a.lane_merge, which the autotuner tries).
// lane heads of at most 8 members in registers: 4,096-graph batch 40.27 ->
// 39.65 ms with the binary search (the merge unchanged), R-MAT unchanged
#ifndef XT_LANE_REGS
#define XT_LANE_REGS 1
#endif
  constexpr int kLaneRegs = 8;
  auto lane_tasks = [&](auto merge_tag) {
    constexpr bool MERGE = decltype(merge_tag)::value;
    // heads are claimed 32 * a.claim at a time (lane 0 keeps the block)
    unsigned long long lnext = 0, lend = 0;
    while (true) {
      unsigned long long base = 0;
      if (lane == 0) {
        if (lnext == lend) {
          lnext = atomicAdd(&cursor[2], 32ull * (unsigned long long)a.claim);
          lend = lnext + 32ull * (unsigned long long)a.claim;
        }
        base = lnext;
        lnext += 32;
      }
      base = __shfl_sync(0xffffffffu, base, 0);
      if (int64_t(base) >= a.n_tt) break;
      const int64_t i = int64_t(base) + lane;
      if (i >= a.n_tt) continue;
      const int32_t v = a.tt[i * a.stride];
      const int64_t r0 = off[v], r1 = off[v + 1];
      const int32_t lo = col[r0], hi = col[r1 - 1];
      // per-edge mode: the counts sit at padded positions; row v's shift
      const int64_t vshift = MODE == 2 ? a.poff[v] - r0 : 0;
      // a head of at most kLaneRegs members (not in the per-edge mode, which
      // needs each hit's position) keeps them in registers: a candidate is
      // then kLaneRegs compares, no dependent load
      const bool regs = XT_LANE_REGS && MODE != 2 && r1 - r0 <= kLaneRegs;
      int32_t mm[kLaneRegs];
#pragma unroll
      for (int j = 0; j < kLaneRegs; j++) mm[j] = (regs && j < r1 - r0) ? col[r0 + j] : -1;
      int64_t hv = 0;
      const int32_t *__restrict__ colp = a.colp;
      for (int64_t k = ioff[v]; k < ioff[v + 1]; k++) {
        const InRec r = rec[k];
        const int64_t rs = rec_s(r), re = rs + rec_len(r);
        const int32_t ru = MODE == 1 ? a.rec_u[k] : 0;
        int64_t b = r0;  // members below b are below every remaining candidate
        int32_t hu = 0;
        for (int64_t p = rs; p < re; p++) {
          const int32_t w = colp[p];
          if (w > hi) break;  // the suffix ascends
          if (w < lo) continue;
          int64_t x = b;
          bool hit;
          if (regs) {
            hit = false;
#pragma unroll
            for (int j = 0; j < kLaneRegs; j++) hit |= w == mm[j];
          } else if (MERGE) {
            while (col[x] < w) x++;  // stops by r1 - 1: w <= hi
          } else {
            int64_t y = r1;
            while (x < y) {
              const int64_t mid = (x + y) >> 1;
              if (col[mid] < w) x = mid + 1;
              else y = mid;
            }
          }
          if (!regs) {
            b = x;
            hit = col[x] == w;  // x < r1: w <= hi
          }
          if (hit) {
            hu++;
            if (MODE == 1) atomicAdd(reinterpret_cast<unsigned long long *>(&pv[w]), 1ull);
            if (MODE == 2) {
              atomicAdd(&es[p], 1u);  // the edge u->w
              atomicAdd(&es[x + vshift], 1u);  // the edge v->w
            }
            if (!regs) b = x + 1;
          }
        }
        hv += hu;
        if (MODE == 1 && hu) atomicAdd(reinterpret_cast<unsigned long long *>(&pv[ru]), (unsigned long long)hu);
        if (MODE == 2 && hu) atomicAdd(&es[rs - 1], unsigned(hu));  // the edge u->v
      }
      acc += hv;
      if (hv) {
        if (MODE == 1) atomicAdd(reinterpret_cast<unsigned long long *>(&pv[v]), (unsigned long long)hv);
        if (a.group) atomicAdd(&a.group_out[a.group[v]], (unsigned long long)hv);
      }
    }
  };
  if (a.lane_merge) lane_tasks(std::true_type{});
  else lane_tasks(std::false_type{});

  // ---- reduce ----
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __syncthreads();
  if (lane == 0) s_red[warp] = (unsigned long long)acc;
  __syncthreads();
  if (tid == 0) {
    unsigned long long tot = 0;
    for (int w = 0; w < kWarps; w++) tot += s_red[w];
    atomicAdd(a.global, tot);
  }
}

// dynamic shared memory: member words; in modes 1 and 2 also hash counters
// or bitmap word starts, and bitmap member counters
// ---- the cluster tier (global count) ---------------------------------------
//
// A cluster of kCluster CTAs counts one cluster task at a time: the part's
// members (up to kClusterDmax, ascending) are split into kCluster contiguous
// runs, CTA c hashing run c into its own table, and every candidate is
// looked up in the table of the CTA whose id range holds it, through
// distributed shared memory. CTA 0 claims each task and publishes it, and a
// cursor for the task's record batches, in its shared memory (two buffers,
// so it can publish the next task while the others still stream the
// current one); all CTAs of the cluster read the same task sequence, so
// they reach the same cluster barriers and leave together when it is empty.
// Counts: warp shuffles, the CTA's warps, then the cluster's CTAs summed in
// CTA 0's shared memory, one global add per cluster.
// record batches: every kCluster-th batch of the task from each CTA's own
// cursor (781 ms on the graph above) or all from one cursor in CTA 0's shared
// memory (823 ms)
#ifndef XT_CLUSTER_SHARED_CURSOR
#define XT_CLUSTER_SHARED_CURSOR 0
#endif
// 4 CTAs of 256 threads per SM (64 registers): Chung-Lu n=4.19M under the id
// orientation 704 ms, against 781 ms at 2 and 784 ms at 3
#ifndef XT_CLUSTER_MINB
#define XT_CLUSTER_MINB 4
#endif
__global__ void __cluster_dims__(kCluster, 1, 1) __launch_bounds__(kThreads, XT_CLUSTER_MINB)
    k_count_cluster(const CountArgs a) {
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  const unsigned rank = cluster.block_rank();
  extern __shared__ int32_t smem[];
  int32_t *table = smem;  // kBlockWords slots
  __shared__ Task s_ct[2];
  __shared__ int s_cbatch[2];
  __shared__ unsigned long long s_cred[kCluster];
  __shared__ unsigned long long s_wred[kWarps];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int32_t *__restrict__ col = a.col;
  const Task *ct0 = cluster.map_shared_rank(s_ct, 0);
  int *cb0 = cluster.map_shared_rank(s_cbatch, 0);
  unsigned long long *red0 = cluster.map_shared_rank(s_cred, 0);
  int lg = 6;
  while ((2 << lg) <= kBlockWords) lg++;
  int64_t acc = 0;
  for (int cur = 0;; cur ^= 1) {
    if (rank == 0 && tid == 0) {
      const unsigned long long i = atomicAdd(&a.cursor[3], 1ull);
      Task t;
      if (int64_t(i) < a.n_ct) {
        t = a.ct[int64_t(i) * a.stride];
      } else {
        t.k0 = t.r0 = 0;
        t.v = t.nmem = t.lg_s = 0;
        t.nrec = -1;
      }
      s_ct[cur] = t;
    }
    if (tid == 0) s_cbatch[cur] = 0;
    cluster.sync();  // the task is published, and every CTA is done with the previous one
    const Task t = ct0[cur];
    if (t.nrec < 0) break;
    // this CTA's run of the part's members into its table
    const int per = (t.nmem + kCluster - 1) / kCluster;
    const int m0 = min(t.nmem, int(rank) * per), m1 = min(t.nmem, m0 + per);
    for (int i = 4 * tid; i < kBlockWords; i += 4 * kThreads)
      *reinterpret_cast<int4 *>(table + i) = make_int4(kEmpty, kEmpty, kEmpty, kEmpty);
    __syncthreads();
    Members m;
    m.words = table;
    m.idx = nullptr;
    m.mcnt = nullptr;
    m.mask = (1u << lg) - 1;
    m.shift = 32 - lg;
    m.base = m.nwords = 0;
    m.bitmap = m.cuckoo = false;
    m.ctab = smem_u32(table);
    for (int i = m0 + tid; i < m1; i += kThreads) hash_insert(table, m.mask, m.shift, col[t.r0 + i]);
    m.lo = col[t.r0];
    m.hi = col[t.r0 + t.nmem - 1];
#pragma unroll
    for (int c = 1; c < kCluster; c++) m.cb[c - 1] = c * per < t.nmem ? col[t.r0 + c * per] : 0x7fffffff;
    cluster.sync();  // every table is built
#if XT_CLUSTER_SHARED_CURSOR
    const int64_t h = stream_kind<0, kKindCluster, false>(a.rec, nullptr, a.colp, t.k0, t.k0 + t.nrec, t.lg_s, cb0 + cur, m,
                                                          nullptr, nullptr, a.off, a.poff, lane);
#else
    const int64_t h = stream_kind<0, kKindCluster, false>(a.rec, nullptr, a.colp, t.k0, t.k0 + t.nrec, t.lg_s, s_cbatch + cur,
                                                          m, nullptr, nullptr, a.off, a.poff, lane, kCluster, rank);
#endif
    acc += h;
    if (a.group) credit_group(a, t.v, h, lane);
  }
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) s_wred[warp] = (unsigned long long)acc;
  __syncthreads();
  if (tid == 0) {
    unsigned long long tot = 0;
    for (int w = 0; w < kWarps; w++) tot += s_wred[w];
    red0[rank] = tot;
  }
  cluster.sync();  // every CTA's sum is in CTA 0
  if (rank == 0 && tid == 0) {
    unsigned long long tot = 0;
    for (int r = 0; r < kCluster; r++) tot += s_cred[r];
    if (tot) atomicAdd(a.global, tot);
  }
}

static size_t count_smem_bytes(bool pv) {
  return pv ? sizeof(int32_t) * (kBlockWords + kBlockDmax) + sizeof(uint16_t) * kBlockWords
            : sizeof(int32_t) * kBlockWords;
}

// per-vertex counts in internal numbering -> input numbering
__global__ void k_unpermute(const int64_t *__restrict__ in, const int32_t *__restrict__ n2o, int64_t nv,
                            int64_t *__restrict__ out) {
  XT_GRID_STRIDE(r, nv) out[n2o[r]] = in[r];
}

// ---- host side --------------------------------------------------------------

static xt_status exclusive_scan(Ctx *c, const int64_t *in, int64_t *out, int64_t n) {
  size_t bytes = 0;
  XT_CUDA(c, cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, c->stream));
  void *tmp = nullptr;
  XT_TRY(dalloc(c, &tmp, bytes));
  cudaError_t e = cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, n, c->stream);
  dfree(c, tmp);
  XT_CUDA(c, e);
  return XT_OK;
}

void free_plan(Graph *g) {
  if (!g->plan) return;
  Ctx *c = g->ctx;
  dfree(c, g->plan->d_bt);
  dfree(c, g->plan->d_ct);
  dfree(c, g->plan->d_bt0);
  dfree(c, g->plan->d_wt);
  dfree(c, g->plan->d_tt);
  dfree(c, g->plan->d_cursor);
  delete g->plan;
  g->plan = nullptr;
}

static xt_status d2h(Ctx *c, void *h, const void *d, size_t bytes) {
  return cuda_status(c, cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, c->stream), "D2H");
}

// The cluster tasks (d_ct) and the CTA tasks of the other heads (d_bt0,
// chunk-major order kept), and the cluster kernel's persistent grid.
static xt_status plan_cluster(Ctx *c, Graph *g, Plan *pl, const int64_t *P, const PlanParams &pp) {
  const int64_t nv = g->nv;
  const int B = 256;
  int64_t *nc = nullptr, *ncp = nullptr, *d_num = nullptr;
  void *tmp = nullptr;
  xt_status s = XT_OK;
  do {
    if ((s = dalloc_n(c, &nc, size_t(nv + 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &ncp, size_t(nv + 1))) != XT_OK) break;
    k_plan_ccount<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(nv, g->d_off, g->d_ioff, P, pp, nc);
    if ((s = cuda_status(c, cudaMemsetAsync(nc + nv, 0, sizeof(int64_t), c->stream), "memset")) != XT_OK) break;
    if ((s = exclusive_scan(c, nc, ncp, nv + 1)) != XT_OK) break;
    int64_t n = 0;
    if ((s = d2h(c, &n, ncp + nv, sizeof(int64_t))) != XT_OK) break;
    if ((s = cuda_status(c, cudaStreamSynchronize(c->stream), "sync")) != XT_OK) break;
    if (n == 0) break;
    if ((s = dalloc_n(c, &pl->d_ct, size_t(n))) != XT_OK) break;
    k_plan_cfill<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(nv, g->d_off, g->d_ioff, P, pp, ncp,
                                                                                pl->d_ct);
    if ((s = cuda_status(c, cudaGetLastError(), "k_plan_cfill")) != XT_OK) break;
    if ((s = dalloc_n(c, &pl->d_bt0, size_t(pl->n_btask))) != XT_OK) break;
    if ((s = dalloc_n(c, &d_num, 1)) != XT_OK) break;
    size_t bytes = 0;
    const NotClusterHead keep{g->d_off};
    if ((s = cuda_status(c, cub::DeviceSelect::If(nullptr, bytes, pl->d_bt, pl->d_bt0, d_num, pl->n_btask, keep,
                                                  c->stream), "task select")) != XT_OK)
      break;
    if ((s = dalloc(c, &tmp, bytes)) != XT_OK) break;
    if ((s = cuda_status(c, cub::DeviceSelect::If(tmp, bytes, pl->d_bt, pl->d_bt0, d_num, pl->n_btask, keep,
                                                  c->stream), "task select")) != XT_OK)
      break;
    int64_t n0 = 0;
    if ((s = d2h(c, &n0, d_num, sizeof(int64_t))) != XT_OK) break;
    if ((s = cuda_status(c, cudaStreamSynchronize(c->stream), "sync")) != XT_OK) break;
    // persistent grid: every cluster that fits on the device at once
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kCluster);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = sizeof(int32_t) * kBlockWords;
    int clusters = 0;
    if ((s = cuda_status(c, cudaOccupancyMaxActiveClusters(&clusters, k_count_cluster, &cfg), "cluster occupancy")) !=
        XT_OK)
      break;
    if (clusters < 1) {
      s = set_error(c, XT_ERR_CUDA, "no thread-block cluster of the cluster tier fits on this device");
      break;
    }
    pl->n_ctask = n;
    pl->n_btask0 = n0;
    pl->grid_cluster = kCluster * int(std::min<int64_t>(clusters, n));
  } while (0);
  dfree(c, nc);
  dfree(c, ncp);
  dfree(c, d_num);
  dfree(c, tmp);
  return s;
}

xt_status make_plan(Graph *g) {
  Ctx *c = g->ctx;
  free_plan(g);
  Plan *pl = new Plan();
  g->plan = pl;
  const int64_t nv = g->nv, ne = g->ne;
  const int B = 256;
  int64_t *P = nullptr, *nb = nullptr, *nw = nullptr, *nt = nullptr, *nbp = nullptr, *nwp = nullptr,
          *ntp = nullptr;
  unsigned long long *stats = nullptr;
  xt_status s = XT_OK;
  do {
    if ((s = dalloc_n(c, &pl->d_cursor, 4)) != XT_OK) break;
    if ((s = dalloc_n(c, &stats, 4)) != XT_OK) break;
    if ((s = dalloc_n(c, &P, size_t(ne + 1))) != XT_OK) break;
    if ((s = cuda_status(c, cudaMemsetAsync(stats, 0, 4 * sizeof(unsigned long long), c->stream), "memset")) !=
        XT_OK)
      break;
    k_vertex_stats<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(g->d_off, g->d_ioff, nv, stats);
    // suffix lengths, prefix-summed in head order
    {
      const auto lens = thrust::make_transform_iterator(thrust::counting_iterator<int64_t>(0), RecLen{g->d_irec, ne});
      size_t bytes = 0;
      if ((s = cuda_status(c, cub::DeviceScan::ExclusiveSum(nullptr, bytes, lens, P, ne + 1, c->stream), "scan")) !=
          XT_OK)
        break;
      void *tmp = nullptr;
      if ((s = dalloc(c, &tmp, bytes)) != XT_OK) break;
      s = cuda_status(c, cub::DeviceScan::ExclusiveSum(tmp, bytes, lens, P, ne + 1, c->stream), "scan");
      dfree(c, tmp);
      if (s != XT_OK) break;
    }
    // persistent grids: every CTA that fits on the device at once
    int occ[3] = {0, 0, 0};
    for (int mode = 0; mode < 3 && s == XT_OK; mode++) {
      auto fn = mode == 0 ? k_count<0, false> : (mode == 1 ? k_count<1, false> : k_count<2, false>);
      const size_t bytes = count_smem_bytes(mode != 0);
      s = cuda_status(c, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)), "attr");
      if (s == XT_OK)
        s = cuda_status(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[mode], fn, kThreads, bytes), "occ");
    }
    if (s == XT_OK)
      s = cuda_status(c, cudaFuncSetAttribute(k_count<0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              int(count_smem_bytes(false))), "attr");
    if (s != XT_OK) break;
    pl->grid_global = c->sm_count * (occ[0] > 0 ? occ[0] : 1);
    pl->grid_pv = c->sm_count * (occ[1] > 0 ? occ[1] : 1);
    pl->grid_es = c->sm_count * (occ[2] > 0 ? occ[2] : 1);
    // CTA task size: large tasks amortise the member-set build and the task
    // barrier, but every CTA should still get about 16 of them
    int64_t total_work = 0;
    if ((s = d2h(c, &total_work, P + ne, sizeof(int64_t))) != XT_OK) break;
    if ((s = cuda_status(c, cudaStreamSynchronize(c->stream), "sync")) != XT_OK) break;
    PlanParams pp;
    pp.warp_dmax = kWarpDmax;
    // graphs of 2^34 or more candidates (R-MAT s24 has 2^35.3) take larger
    // warp tasks and more record batches per warp
    const bool large = total_work >= (int64_t(1) << 34);
    // lane tasks trade latency (a lane's dependent loads set the kernel's
    // tail) for throughput: only graphs with plenty of other work use them
    pp.tiny_work = total_work >= (int64_t(1) << 30) ? XT_TINY_WORK : 0;
    if (g->tier_lane_work >= 0) pp.tiny_work = g->tier_lane_work;
    pp.batches_per_warp = large ? XT_BATCHES_PER_WARP_LARGE : XT_BATCHES_PER_WARP;
    pp.lane_pairs = XT_LANE_PAIRS;
    pp.warp_work = g->tune_warp_work > 0 ? g->tune_warp_work : (large ? XT_WARP_WORK_LARGE : kWarpWork);
    if (g->tier_warp_work >= 0) pp.warp_work = g->tier_warp_work;
    if (g->tune_block_work > 0) {
      pp.block_work = g->tune_block_work;
    } else {
      pp.block_work = kBlockWorkMin;
      while (pp.block_work < kBlockWorkMax && pp.block_work * 16 * pl->grid_global < total_work) pp.block_work *= 2;
    }
    pl->block_work = pp.block_work;
    pl->warp_work = pp.warp_work;
    pl->bitmap_bits = g->tune_bitmap_bits > 0 ? g->tune_bitmap_bits : int64_t(kBlockWords) * 32;
    if ((s = dalloc_n(c, &nb, size_t(nv + 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &nw, size_t(nv + 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &nbp, size_t(nv + 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &nwp, size_t(nv + 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &nt, size_t(nv + 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &ntp, size_t(nv + 1))) != XT_OK) break;
    k_plan_count<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(nv, g->d_off, g->d_ioff, P, pp, nb,
                                                                                nw, nt);
    if ((s = cuda_status(c, cudaMemsetAsync(nb + nv, 0, sizeof(int64_t), c->stream), "memset")) != XT_OK) break;
    if ((s = cuda_status(c, cudaMemsetAsync(nw + nv, 0, sizeof(int64_t), c->stream), "memset")) != XT_OK) break;
    if ((s = cuda_status(c, cudaMemsetAsync(nt + nv, 0, sizeof(int64_t), c->stream), "memset")) != XT_OK) break;
    if ((s = exclusive_scan(c, nb, nbp, nv + 1)) != XT_OK) break;
    if ((s = exclusive_scan(c, nw, nwp, nv + 1)) != XT_OK) break;
    if ((s = exclusive_scan(c, nt, ntp, nv + 1)) != XT_OK) break;
    int64_t h[4] = {0, 0, 0, 0};
    unsigned long long hs[4] = {0, 0, 0, 0};
    if ((s = d2h(c, &h[0], nbp + nv, sizeof(int64_t))) != XT_OK) break;
    if ((s = d2h(c, &h[1], nwp + nv, sizeof(int64_t))) != XT_OK) break;
    if ((s = d2h(c, &h[2], P + ne, sizeof(int64_t))) != XT_OK) break;
    if ((s = d2h(c, &h[3], ntp + nv, sizeof(int64_t))) != XT_OK) break;
    if ((s = d2h(c, hs, stats, sizeof(hs))) != XT_OK) break;
    if ((s = cuda_status(c, cudaStreamSynchronize(c->stream), "sync")) != XT_OK) break;
    pl->n_btask = h[0];
    pl->n_wtask = h[1];
    pl->n_ttask = h[3];
    g->max_degree = int64_t(hs[0]);
    g->max_out_degree = int64_t(hs[1]);
    g->max_in_degree = int64_t(hs[2]);
    g->wedge_work = int64_t(hs[3]);
    g->stream_work = h[2];
    if (g->max_out_degree >= kMaxOutDegree) {
      s = set_error(c, XT_ERR_OVERFLOW, "an oriented out-degree of 2^29 or more is not supported");
      break;
    }
    if ((s = dalloc_n(c, &pl->d_bt, size_t(pl->n_btask > 0 ? pl->n_btask : 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &pl->d_wt, size_t(pl->n_wtask > 0 ? pl->n_wtask : 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &pl->d_tt, size_t(pl->n_ttask > 0 ? pl->n_ttask : 1))) != XT_OK) break;
    k_plan_fill<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(
        nv, g->d_off, g->d_ioff, P, pp, nbp, nwp, ntp, pl->d_bt, pl->d_wt, pl->d_tt);
    if ((s = cuda_status(c, cudaGetLastError(), "k_plan_fill")) != XT_OK) break;
    if (pl->n_btask > 1) {  // chunk-major order
      uint64_t *k1 = nullptr, *k2 = nullptr;
      int32_t *i1 = nullptr, *i2 = nullptr;
      Task *tmp = nullptr;
      void *tb = nullptr;
      const int64_t nt = pl->n_btask;
      size_t bytes = 0;
      s = dalloc_n(c, &k1, size_t(nt));
      if (s == XT_OK) s = dalloc_n(c, &k2, size_t(nt));
      if (s == XT_OK) s = dalloc_n(c, &i1, size_t(nt));
      if (s == XT_OK) s = dalloc_n(c, &i2, size_t(nt));
      if (s == XT_OK) s = dalloc_n(c, &tmp, size_t(nt));
      if (s == XT_OK) {
        k_task_keys<<<counted(c, grid_for(nt, B, c->sm_count)), B, 0, c->stream>>>(pl->d_bt, nt, nbp, k1, i1);
        s = cuda_status(c, cub::DeviceRadixSort::SortPairs(nullptr, bytes, k1, k2, i1, i2, nt, 0, 64, c->stream),
                        "task order");
      }
      if (s == XT_OK) s = dalloc(c, &tb, bytes);
      if (s == XT_OK)
        s = cuda_status(c, cub::DeviceRadixSort::SortPairs(tb, bytes, k1, k2, i1, i2, nt, 0, 64, c->stream),
                        "task order");
      if (s == XT_OK) {
        k_task_gather<<<counted(c, grid_for(nt, B, c->sm_count)), B, 0, c->stream>>>(pl->d_bt, i2, nt, tmp);
        s = cuda_status(c, cudaMemcpyAsync(pl->d_bt, tmp, sizeof(Task) * nt, cudaMemcpyDeviceToDevice, c->stream),
                        "task order");
      }
      dfree(c, tb);
      dfree(c, k1);
      dfree(c, k2);
      dfree(c, i1);
      dfree(c, i2);
      dfree(c, tmp);
    }
    if (s != XT_OK) break;
    // global count: heads whose members overflow a CTA's set go to the
    // cluster tier instead of CTA tasks over parts of their members
    if (g->cluster_tier != 0 && g->max_out_degree > kBlockDmax && pl->n_btask > 0)
      s = plan_cluster(c, g, pl, P, pp);
  } while (0);
  dfree(c, P);
  dfree(c, nb);
  dfree(c, nw);
  dfree(c, nbp);
  dfree(c, nwp);
  dfree(c, nt);
  dfree(c, ntp);
  dfree(c, stats);
  if (s != XT_OK) free_plan(g);
  return s;
}

int64_t cluster_task_count(const Graph *g) { return g->plan ? g->plan->n_ctask : 0; }
int64_t lane_task_count(const Graph *g) { return g->plan ? g->plan->n_ttask : 0; }

// After a count has finished on the context stream: XT_ERR_TIMEOUT if a
// CTA's bounded wait for its staged members gave up (the count is then
// incomplete), which clears the flag; XT_OK otherwise.
xt_status count_status(Ctx *c) {
  int h = 0;
  XT_CUDA(c, cudaMemcpyAsync(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  XT_CUDA(c, cudaStreamSynchronize(c->stream));
  if (h & kErrStageTimeout) {
    XT_CUDA(c, cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
    return set_error(c, XT_ERR_TIMEOUT, "count: a CTA's wait for its staged member list timed out");
  }
  return XT_OK;
}

// the tail u of each in-record: the row whose padded span holds position
// s - 1 (the head's own column in N+(u)); the last row starting at or before
// it is that row, as an empty row starts where the next one does
__global__ void k_rec_tails(const InRec *__restrict__ rec, int64_t ne, const int64_t *__restrict__ poff, int64_t nv,
                            int32_t *__restrict__ u) {
  XT_GRID_STRIDE(e, ne) {
    const int64_t q = rec_s(rec[e]) - 1;
    int64_t lo = 0, hi = nv;  // poff[lo] <= q < poff[hi]
    while (hi - lo > 1) {
      const int64_t mid = (lo + hi) >> 1;
      if (poff[mid] <= q) lo = mid;
      else hi = mid;
    }
    u[e] = int32_t(lo);
  }
}

// per-edge counts from padded positions (row u at poff[u]) to the out-CSR's
// (row u at off[u]), widened to 64 bits: a warp per row
__global__ void k_es_unpad(const unsigned int *__restrict__ esp, const int64_t *__restrict__ off,
                           const int64_t *__restrict__ poff, int64_t nv, int64_t *__restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t u = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; u < nv; u += nw) {
    const int64_t r0 = off[u], len = off[u + 1] - r0, p0 = poff[u];
    for (int64_t i = lane; i < len; i += 32) out[r0 + i] = int64_t(esp[p0 + i]);
  }
}

// tasks of a list of n that fall to shard `shard` of nshards (every
// nshards-th, from index shard on)
static int64_t shard_len(int64_t n, int shard, int nshards) {
  return n > shard ? (n - shard + nshards - 1) / nshards : 0;
}
// the shard's first task of a list of n (null when the shard has none)
template <typename T>
static const T *shard_first(const T *p, int64_t n, int shard) {
  return p && n > shard ? p + shard : nullptr;
}

xt_status count_graph(Graph *g, int64_t *d_global, int64_t *d_pv, int64_t *d_groups, int64_t *d_support, int shard,
                      int nshards) {
  Ctx *c = g->ctx;
  if (nshards < 1 || shard < 0 || shard >= nshards)
    return set_error(c, XT_ERR_INVALID, "shard must lie in [0, nshards) and nshards be at least 1");
  if (!g->plan) XT_TRY(make_plan(g));
  Plan *pl = g->plan;
  // pairs of columns are read with 32-byte vector loads
  if (reinterpret_cast<uintptr_t>(g->d_colp) % 32 != 0)
    return set_error(c, XT_ERR_CUDA, "padded column array is not 32-byte aligned");
  XT_CUDA(c, cudaMemsetAsync(pl->d_cursor, 0, 4 * sizeof(unsigned long long), c->stream));
  XT_CUDA(c, cudaMemsetAsync(d_global, 0, sizeof(int64_t), c->stream));
  if (d_groups) {
    if (!g->d_group) return set_error(c, XT_ERR_INVALID, "per-group counts need a graph built as a batch");
    XT_CUDA(c, cudaMemsetAsync(d_groups, 0, sizeof(int64_t) * g->n_groups, c->stream));
  }
  if (d_pv && d_support) return set_error(c, XT_ERR_INVALID, "per-vertex and per-edge counts are separate calls");
  // per-edge counts, 32-bit while counting, at the padded column positions
  // (a record's suffix and its tail's edge are found there without the
  // tail's row offsets)
  unsigned int *es = nullptr;
  if (d_support) {
    const size_t n = size_t(g->colp_len > 0 ? g->colp_len : 1);
    XT_TRY(dalloc_n(c, &es, n));
    XT_CUDA(c, cudaMemsetAsync(es, 0, sizeof(unsigned int) * n, c->stream));
  }
  if (d_pv && !g->d_irec_u && g->ne > 0) {  // the records' tails, once per graph
    XT_TRY(dalloc_n(c, &g->d_irec_u, size_t(g->ne)));
    k_rec_tails<<<counted(c, grid_for(g->ne, 256, c->sm_count)), 256, 0, c->stream>>>(g->d_irec, g->ne, g->d_poff,
                                                                                      g->nv, g->d_irec_u);
    XT_CUDA(c, cudaGetLastError());
  }
  int64_t *pv_int = nullptr;  // per-vertex counts in internal numbering
  if (d_pv) {
    if (g->d_perm) XT_TRY(dalloc_n(c, &pv_int, size_t(g->nv)));
    else pv_int = d_pv;
    XT_CUDA(c, cudaMemsetAsync(pv_int, 0, sizeof(int64_t) * g->nv, c->stream));
  }
  CountArgs a;
  a.off = g->d_off;
  a.col = g->d_col;
  a.colp = g->d_colp;
  a.poff = g->d_poff;
  a.ioff = g->d_ioff;
  a.rec = g->d_irec;
  a.rec_u = g->d_irec_u;
  a.bt = shard_first(pl->d_bt, pl->n_btask, shard);
  a.n_bt = shard_len(pl->n_btask, shard, nshards);
  a.wt = shard_first(pl->d_wt, pl->n_wtask, shard);
  a.n_wt = shard_len(pl->n_wtask, shard, nshards);
  a.tt = shard_first(pl->d_tt, pl->n_ttask, shard);
  a.n_tt = shard_len(pl->n_ttask, shard, nshards);
  a.ct = shard_first(pl->d_ct, pl->n_ctask, shard);
  a.n_ct = shard_len(pl->n_ctask, shard, nshards);
  a.stride = nshards;
  a.claim = g->claim_block > 0 ? g->claim_block : (g->n_groups > 0 ? 4 : 1);
  a.lane_merge = g->lane_merge;
  a.cursor = pl->d_cursor;
  a.global = reinterpret_cast<unsigned long long *>(d_global);
  a.pv = pv_int;
  a.es = es;
  a.group = d_groups ? g->d_group : nullptr;
  a.group_out = reinterpret_cast<unsigned long long *>(d_groups);
  a.bitmap_bits = pl->bitmap_bits;
  a.cuckoo_iters = g->cuckoo_iters >= 0 ? g->cuckoo_iters : kCuckooIters;
  a.err = c->d_err;
  if (g->ne > 0) {
    if (d_support)
      k_count<2, false><<<counted(c, pl->grid_es), kThreads, count_smem_bytes(true), c->stream>>>(a);
    else if (d_pv)
      k_count<1, false><<<counted(c, pl->grid_pv), kThreads, count_smem_bytes(true), c->stream>>>(a);
    else {
      // cluster heads leave the CTA task list to the cluster tier
      CountArgs a0 = a;
      if (pl->n_ctask > 0) {
        a0.bt = shard_first(pl->d_bt0, pl->n_btask0, shard);
        a0.n_bt = shard_len(pl->n_btask0, shard, nshards);
      }
      if (g->prefetch_suffix > 0)
        k_count<0, true><<<counted(c, pl->grid_global), kThreads, count_smem_bytes(false), c->stream>>>(a0);
      else
        k_count<0, false><<<counted(c, pl->grid_global), kThreads, count_smem_bytes(false), c->stream>>>(a0);
      if (pl->n_ctask > 0)
        k_count_cluster<<<counted(c, dim3(pl->grid_cluster)), kThreads, sizeof(int32_t) * kBlockWords, c->stream>>>(a);
    }
  }
  if (d_support && g->ne > 0)
    k_es_unpad<<<counted(c, grid_for(g->nv * 32, 256, c->sm_count)), 256, 0, c->stream>>>(es, g->d_off, g->d_poff,
                                                                                          g->nv, d_support);
  if (d_pv && g->d_perm)
    k_unpermute<<<counted(c, grid_for(g->nv, 256, c->sm_count)), 256, 0, c->stream>>>(pv_int, g->d_perm, g->nv, d_pv);
  cudaError_t e = cudaGetLastError();
  if (pv_int && pv_int != d_pv) dfree(c, pv_int);
  dfree(c, es);
  XT_CUDA(c, e);
  return XT_OK;
}

}  // namespace xt
