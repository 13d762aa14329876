// Degree-binned schedule and the exact triangle-count kernel.
//
// Vertices are numbered by orientation rank (see build.cu), so every triangle
// {u,v,w} with u < v < w is the edges u->v, u->w, v->w. The reference finds it
// from the lowest corner i=u: for every pair m < n of its sorted row it
// binary-searches adj(v) for w (xxtric.hpp:150-207, check_edgelist
// xxtric.hpp:516-545). Here it is found from the MIDDLE corner v:
//   1. N+(v) is loaded once into shared memory as a membership structure:
//      a bitmap over [min N+(v), max N+(v)] when that range is small enough,
//      else an open-addressing hash table (load factor <= 1/4);
//   2. for every in-edge u->v, the suffix of N+(u) after v (the reference's
//      n > m range) is streamed through it. A candidate below min N+(v) is
//      skipped and one above max N+(v) ends that suffix (the reference's
//      edge_above_min / edge_within_max prunes, xxtric.hpp:576-588).
// Items streamed: sum over u of C(d+(u), 2), each tested in shared memory.
//
// Schedule (make_plan): per head v, work(v) = total suffix length.
//   warp bin : d+(v) <= kWarpDmax and work(v) <= kWarpWork -> one warp per v
//   block bin: otherwise -> CTA tasks over chunks of v's in-records of about
//              kBlockWork items; N+(v) beyond kBlockDmax members is split
//              into parts, one task per (part, chunk)
// One persistent kernel drains the CTA tasks first (the large ones), then the
// warp tasks, each from its own global atomic cursor.
#include <cub/cub.cuh>

#include "xt_internal.cuh"

namespace xt {

// Tuning constants (compile-time; the XT_* macros let a build override them)
#ifndef XT_THREADS
#define XT_THREADS 256
#endif
#ifndef XT_BLOCK_WORK_LOG2
#define XT_BLOCK_WORK_LOG2 20
#endif
#ifndef XT_WARP_WORK
#define XT_WARP_WORK 4096
#endif
constexpr int kThreads = XT_THREADS;
constexpr int kWarps = kThreads / 32;
#ifndef XT_MIN_BLOCKS
#define XT_MIN_BLOCKS (1024 / XT_THREADS)
#endif
constexpr int kMinBlocks = XT_MIN_BLOCKS;  // CTAs per SM the register budget is sized for
constexpr int kWarpDmax = 64;
constexpr int kWarpWords = 256;   // per-warp region: 256-slot hash or 8192-bit bitmap
constexpr int64_t kWarpWork = XT_WARP_WORK;
constexpr int kBlockDmax = 2048;
constexpr int kBlockWords = 8192;  // CTA region: 8192-slot hash or 2^18-bit bitmap
constexpr int64_t kBlockWorkMin = int64_t(1) << 14;
constexpr int64_t kBlockWorkMax = int64_t(1) << XT_BLOCK_WORK_LOG2;

// Run-time schedule thresholds (the binning of make_plan).
struct PlanParams {
  int64_t warp_work;   // a head with d+(v) <= warp_dmax and at most this much work is a warp task
  int64_t block_work;  // items per CTA task
  int32_t warp_dmax;
};
constexpr int32_t kEmpty = -1;

struct Plan {
  int64_t n_btask = 0;        // CTA tasks
  int64_t *d_bt = nullptr;    // 4 int64 per task: v, part, k0, k1 (k = in-record index)
  int64_t n_wtask = 0;        // warp tasks
  int32_t *d_wt = nullptr;    // v per warp task
  unsigned long long *d_cursor = nullptr;  // [0] CTA cursor, [1] warp cursor
  int grid_global = 0, grid_pv = 0;
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

__global__ void k_inrec_work(const InRec *__restrict__ rec, int64_t ne, int64_t *__restrict__ w) {
  XT_GRID_STRIDE(e, ne) w[e] = rec[e].len;
}

// tail-grouped work (statistics): d+(col[e]) per out-edge
__global__ void k_outedge_work(const int32_t *__restrict__ col, int64_t ne, const int64_t *__restrict__ off,
                               int64_t *__restrict__ w) {
  XT_GRID_STRIDE(e, ne) {
    const int32_t v = col[e];
    w[e] = off[v + 1] - off[v];
  }
}

__device__ __forceinline__ void classify(int64_t v, const int64_t *__restrict__ off, const int64_t *__restrict__ ioff,
                                         const int64_t *__restrict__ P, const PlanParams pp, int64_t &nb,
                                         int64_t &nw, int64_t &parts, int64_t &chunks, int64_t &work) {
  const int64_t dp = off[v + 1] - off[v];
  const int64_t k0 = ioff[v], k1 = ioff[v + 1];
  nb = nw = parts = chunks = 0;
  work = P[k1] - P[k0];
  if (dp == 0 || work == 0) return;
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
                             int64_t *__restrict__ nw_out) {
  XT_GRID_STRIDE(v, nv) {
    int64_t nb, nw, parts, chunks, work;
    classify(v, off, ioff, P, pp, nb, nw, parts, chunks, work);
    nb_out[v] = nb;
    nw_out[v] = nw;
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

__global__ void k_plan_fill(int64_t nv, const int64_t *__restrict__ off, const int64_t *__restrict__ ioff,
                            const int64_t *__restrict__ P, const PlanParams pp, const int64_t *__restrict__ nb_pos,
                            const int64_t *__restrict__ nw_pos, int64_t *__restrict__ bt, int32_t *__restrict__ wt) {
  XT_GRID_STRIDE(v, nv) {
    int64_t nb, nw, parts, chunks, work;
    classify(v, off, ioff, P, pp, nb, nw, parts, chunks, work);
    if (nw) wt[nw_pos[v]] = int32_t(v);
    if (!nb) continue;
    const int64_t k0 = ioff[v], k1 = ioff[v + 1], base = P[k0];
    int64_t t = nb_pos[v], prev = k0;
    for (int64_t c = 0; c < chunks; c++) {
      const int64_t kend = (c + 1 == chunks) ? k1 : lower_bound_i64(P, prev, k1, base + (work * (c + 1)) / chunks);
      if (kend <= prev) continue;  // empty chunk (one in-record carries more work)
      for (int64_t p = 0; p < parts; p++) {
        bt[4 * t + 0] = v;
        bt[4 * t + 1] = p;
        bt[4 * t + 2] = prev;
        bt[4 * t + 3] = kend;
        t++;
      }
      prev = kend;
    }
    for (; t < nb_pos[v] + nb; t++) {  // slots of empty chunks: no-op tasks
      bt[4 * t + 0] = v;
      bt[4 * t + 1] = 0;
      bt[4 * t + 2] = k1;
      bt[4 * t + 3] = k1;
    }
  }
}

// ---- membership structures --------------------------------------------------

__device__ __forceinline__ uint32_t hash_slot(int32_t x, int shift) {
  return (uint32_t(x) * 0x9E3779B1u) >> shift;
}

__device__ __forceinline__ void hash_insert(int32_t *tab, uint32_t mask, int shift, int32_t x) {
  uint32_t h = hash_slot(x, shift);
  while (true) {
    const int32_t old = atomicCAS(&tab[h], kEmpty, x);
    if (old == kEmpty || old == x) return;
    h = (h + 1) & mask;
  }
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
  int32_t *cnt;     // per-slot hit counters (per-vertex mode, hash only)
  int32_t lo, hi;   // smallest and largest member
  uint32_t mask;    // hash: slots - 1
  int shift;        // hash: 32 - log2(slots)
  bool bitmap;
};

// Chooses the structure for members col[r0, r1) that fits `words` words (a
// bitmap only while the members' id range is at most bitmap_bits) and
// returns how many words must be cleared.
template <bool PV>
__device__ __forceinline__ int members_layout(Members &m, const int32_t *__restrict__ col, int64_t r0, int64_t r1,
                                              int words, int64_t bitmap_bits) {
  m.lo = col[r0];
  m.hi = col[r1 - 1];
  const int64_t range = int64_t(m.hi) - int64_t(m.lo) + 1;
  m.bitmap = !PV && range <= int64_t(words) * 32 && range <= bitmap_bits;
  if (m.bitmap) {
    m.mask = 0;
    m.shift = 0;
    return int((range + 31) >> 5);
  }
  int lg = 6;
  while ((int64_t(1) << lg) < 4 * (r1 - r0)) lg++;  // load factor <= 1/4: an absent key costs ~1.2 probes
  m.mask = (1u << lg) - 1;
  m.shift = 32 - lg;
  return 1 << lg;
}

__device__ __forceinline__ void members_insert(const Members &m, int32_t x) {
  if (m.bitmap) {
    const uint32_t d = uint32_t(x - m.lo);
    atomicOr(reinterpret_cast<unsigned int *>(&m.words[d >> 5]), 1u << (d & 31));
  } else {
    hash_insert(m.words, m.mask, m.shift, x);
  }
}

// ---- streaming the in-record suffixes ----------------------------------------

// A warp step: kStepGroups x 32 aligned 16-byte groups (kStepGroups LDG.128
// per lane) taken from the flattened groups of a batch of suffixes, so a
// step spans as many suffixes as it needs and every lane has groups while
// the batch lasts.
#ifndef XT_STEP_GROUPS
#define XT_STEP_GROUPS 2
#endif
constexpr int kStepGroups = XT_STEP_GROUPS;

struct Chunk {
  int4 x[kStepGroups];     // four columns per group
  uint32_t vm[kStepGroups];  // which of the four are inside the suffix (bit i: column i)
  int32_t rj[kStepGroups];   // the suffix's slot in the batch (per-vertex credit)
  bool exists;               // warp-uniform: this step exists
};

// bits i in [0,4) with pos + i in [lo, hi), where lo - pos <= 3 whenever
// lo > pos (a suffix starts inside its first group)
__device__ __forceinline__ uint32_t valid_mask(uint32_t pos, uint32_t lo, uint32_t hi) {
  const uint32_t a = lo > pos ? lo - pos : 0u;
  uint32_t b = hi > pos ? hi - pos : 0u;
  b = b > 4u ? 4u : b;
  return ((1u << b) - 1u) & ~((1u << a) - 1u);
}

// Per-warp shared-memory view of the current batch.
// Flattened positions are 4 x flattened group + column in group; a batch
// holds at most 32 suffixes of fewer than kMaxOutDegree columns each, so
// positions fit in 32 bits.
constexpr int64_t kMaxOutDegree = int64_t(1) << 27;

struct BatchView {
  uint32_t start[33];  // first flattened group of each suffix; start[32] = total
  int64_t gbase[32];   // first global group index of each suffix, minus its start
  uint32_t lopos[32];  // the suffix's first flattened position
  uint32_t hipos[32];  // one past its last
  int32_t u[32];       // the suffix's owner
  int32_t hits[32];    // per-vertex mode: hits per suffix in this batch
};

// One warp's walk over the in-records rec[k0, kend), taken in batches of bsz
// records (lane j < bsz holds record j of a batch). Batches come one after
// another (a warp task), or from a cursor in shared memory that the warps of
// a CTA task share, so warps that finish early take more. The next batch is
// claimed and its records loaded while the current one streams.
template <bool PV>
struct FlatWalk {
  const InRec *__restrict__ rec;  // the task's records: rec[0, kend)
  const int32_t *__restrict__ col;
  int64_t *__restrict__ pv;
  BatchView *bv;
  int *cursor;                // shared batch cursor (CTA task) or null
  int32_t kend;               // records in the task
  int32_t kb, nkb, seq;       // current / next batch base, next sequential base
  int bsz, nb;
  int4 nrec;                  // lane's record of the next batch (prefetched)
  uint32_t total, F;          // groups in the batch, next step's first group (uniform)
  int r;                      // this lane's suffix cursor (monotone within a batch)
  // this lane's copy of suffix r's layout: flattened groups end at c_end,
  // global group = flattened + c_gb, valid flattened positions [c_lo, c_hi)
  uint32_t c_end, c_lo, c_hi;
  int64_t c_gb;
  bool have;
  int lane;

  __device__ __forceinline__ void load_suffix() {
    c_end = bv->start[r + 1];
    c_gb = bv->gbase[r];
    c_lo = bv->lopos[r];
    c_hi = bv->hipos[r];
  }

  __device__ __forceinline__ int32_t claim() {
    if (!cursor) {
      const int32_t b = seq;
      seq += bsz;
      return b;
    }
    int c = 0;
    if (lane == 0) c = atomicAdd(cursor, bsz);
    return __shfl_sync(0xffffffffu, c, 0);
  }
  __device__ __forceinline__ int4 fetch(int32_t base) const {
    const int32_t k = base + lane;
    return (lane < bsz && k < kend) ? __ldg(reinterpret_cast<const int4 *>(rec) + k) : make_int4(0, 0, 0, -1);
  }
  // per-vertex mode: credit the finished batch's suffix owners
  __device__ __forceinline__ void flush() {
    if (PV && nb > 0) {
      __syncwarp();
      if (lane < nb && bv->hits[lane])
        atomicAdd(reinterpret_cast<unsigned long long *>(&pv[bv->u[lane]]), (unsigned long long)bv->hits[lane]);
    }
  }
  // lays the batch whose records are in lane registers r4 out in shared memory
  __device__ __forceinline__ void take(int4 r4) {
    flush();
    const int64_t s = int64_t(uint32_t(r4.x)) | (int64_t(r4.y) << 32);
    const uint32_t len = uint32_t(r4.z);
    const int64_t g0 = s >> 2;
    const uint32_t ng = (len > 0) ? uint32_t(((s + len + 3) >> 2) - g0) : 0u;
    uint32_t incl = ng;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    total = __shfl_sync(0xffffffffu, incl, 31);
    __syncwarp();  // every lane is done reading the previous batch
    const uint32_t st = incl - ng;
    bv->start[lane] = st;
    if (lane == 31) bv->start[32] = incl;
    bv->gbase[lane] = g0 - int64_t(st);
    bv->lopos[lane] = 4u * st + uint32_t(s & 3);
    bv->hipos[lane] = 4u * st + uint32_t(s & 3) + len;
    if (PV) {
      bv->u[lane] = r4.w;
      bv->hits[lane] = 0;
    }
    __syncwarp();
    nb = (kend - kb < bsz) ? (kend - kb) : bsz;
    F = 0;
    r = 0;
    load_suffix();
    nkb = claim();
    nrec = fetch(nkb);
  }
  __device__ __forceinline__ void init() {
    nb = 0;
    seq = 0;
    kb = claim();
    have = kb < kend;
    if (have) take(fetch(kb));
  }
  __device__ __forceinline__ Chunk issue() {
    Chunk c;
    while (have && F >= total) {  // batch exhausted: move to the next one
      kb = nkb;
      if (kb >= kend) {
        flush();
        have = false;
        break;
      }
      take(nrec);
    }
    c.exists = have;
#pragma unroll
    for (int q = 0; q < kStepGroups; q++) {
      c.x[q] = make_int4(0, 0, 0, 0);
      c.vm[q] = 0;  // lanes past the batch probe nothing
      c.rj[q] = 0;
    }
    if (!have) return c;
    // this lane's kStepGroups consecutive groups: usually one suffix, so the
    // layout read from shared memory is reused from the previous group
#pragma unroll
    for (int q = 0; q < kStepGroups; q++) {
      const uint32_t f = F + uint32_t(kStepGroups * lane + q);
      if (f < total) {
        if (f >= c_end) {
          do r++;
          while (bv->start[r + 1] <= f);
          load_suffix();
        }
        c.x[q] = __ldg(reinterpret_cast<const int4 *>(col) + (int64_t(f) + c_gb));
        c.vm[q] = valid_mask(4u * f, c_lo, c_hi);
        c.rj[q] = r;
      }
    }
    F += 32 * kStepGroups;
    return c;
  }
};

// Probes one group; returns the hits. A candidate outside
// [min N+(v), max N+(v)] is rejected by one unsigned compare.
template <bool PV, bool BITMAP>
__device__ __forceinline__ int probe_group(int4 x4, uint32_t vm, const Members &m) {
  int h = 0;
  const int32_t w[4] = {x4.x, x4.y, x4.z, x4.w};
  const uint32_t span = uint32_t(m.hi - m.lo);
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const uint32_t d = uint32_t(w[i] - m.lo);
    const bool ok = ((vm >> i) & 1u) && d <= span;
    if (BITMAP) {
      // branch-free: an invalid candidate reads word 0 and is masked out
      const uint32_t word = uint32_t(m.words[ok ? (d >> 5) : 0u]);
      h += int((word >> (d & 31)) & uint32_t(ok));
    } else if (ok) {
      const int slot = hash_find(m.words, m.mask, m.shift, w[i]);
      if (slot >= 0) {
        h++;
        if (PV) atomicAdd(&m.cnt[slot], 1);
      }
    }
  }
  return h;
}

// Streams the suffixes of in-records [k0, kend) in batches of bsz records
// (claimed from `cursor` when it is not null) through the member set;
// returns this lane's hit count.
template <bool PV, bool BITMAP>
__device__ __forceinline__ int64_t stream_kind(const InRec *__restrict__ rec, const int32_t *__restrict__ col,
                                               int64_t k0, int64_t kend, int bsz, int *cursor, const Members &m,
                                               BatchView *bv, int64_t *__restrict__ pv, int lane) {
  FlatWalk<PV> wk;
  wk.rec = rec + k0;
  wk.col = col;
  wk.pv = pv;
  wk.bv = bv;
  wk.cursor = cursor;
  wk.kend = int32_t(kend - k0);
  wk.bsz = bsz;
  wk.lane = lane;
  wk.init();
  int64_t hits = 0;
  Chunk a = wk.issue();
  while (a.exists) {
    Chunk b;
    if (PV) {
      // credit a's suffixes before the next issue may lay a new batch (and
      // flush the credits) over their slots
#pragma unroll
      for (int q = 0; q < kStepGroups; q++) {
        const int h = probe_group<PV, BITMAP>(a.x[q], a.vm[q], m);
        if (h) atomicAdd(&bv->hits[a.rj[q]], h);
        hits += h;
      }
      b = wk.issue();
    } else {
      b = wk.issue();  // the next step's loads are in flight during these probes
      int h = 0;
#pragma unroll
      for (int q = 0; q < kStepGroups; q++) h += probe_group<PV, BITMAP>(a.x[q], a.vm[q], m);
      hits += h;
    }
    a = b;
  }
  return hits;
}

template <bool PV>
__device__ __forceinline__ int64_t stream_suffixes(const InRec *__restrict__ rec, const int32_t *__restrict__ col,
                                                   int64_t k0, int64_t kend, int bsz, int *cursor, const Members &m,
                                                   BatchView *bv, int64_t *__restrict__ pv, int lane) {
  // the membership kind is fixed per task: one specialised loop each
  if (m.bitmap) return stream_kind<PV, true>(rec, col, k0, kend, bsz, cursor, m, bv, pv, lane);
  return stream_kind<PV, false>(rec, col, k0, kend, bsz, cursor, m, bv, pv, lane);
}

// ---- the count kernel ---------------------------------------------------------

struct CountArgs {
  const int64_t *off;
  const int32_t *col;
  const int64_t *ioff;
  const InRec *rec;
  const int64_t *bt;  // CTA tasks
  int64_t n_bt;
  const int32_t *wt;  // warp tasks
  int64_t n_wt;
  unsigned long long *cursor;     // [0] CTA cursor, [1] warp cursor
  unsigned long long *global;     // the total
  int64_t *pv;                    // per-vertex counts (per-vertex mode)
  const int32_t *group;           // head -> group (a graph of a batch), or null
  unsigned long long *group_out;  // per-group counts when group != null
  int64_t bitmap_bits;            // largest member id range kept as a bitmap
};

// adds a warp's hits of one task to the task head's group
__device__ __forceinline__ void credit_group(const CountArgs &a, int64_t v, int64_t h, int lane) {
  for (int o = 16; o; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
  if (lane == 0 && h) atomicAdd(&a.group_out[a.group[v]], (unsigned long long)h);
}

template <bool PV>
__global__ void __launch_bounds__(kThreads, kMinBlocks) k_count(const CountArgs a) {
  const int64_t *__restrict__ off = a.off;
  const int32_t *__restrict__ col = a.col;
  const int64_t *__restrict__ ioff = a.ioff;
  const InRec *__restrict__ rec = a.rec;
  const int64_t *__restrict__ bt = a.bt;
  const int32_t *__restrict__ wt = a.wt;
  const int64_t n_bt = a.n_bt, n_wt = a.n_wt;
  unsigned long long *__restrict__ cursor = a.cursor;
  int64_t *__restrict__ pv = a.pv;
  extern __shared__ int32_t smem[];
  int32_t *bwords = smem;                                   // kBlockWords
  int32_t *bcnt = smem + kBlockWords;                       // kBlockWords (PV only)
  int32_t *wwords_all = smem + (PV ? 2 : 1) * kBlockWords;  // kWarps * kWarpWords
  int32_t *wcnt_all = wwords_all + kWarps * kWarpWords;     // (PV only)
  __shared__ int64_t s_task;
  __shared__ int s_batch;  // next in-record batch of the current CTA task
  __shared__ unsigned long long s_red[kWarps];
  __shared__ BatchView s_bv[kWarps];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int64_t acc = 0;

  // ---- CTA tasks ----
  while (true) {
    if (tid == 0) {
      s_task = int64_t(atomicAdd(&cursor[0], 1ull));
      s_batch = 0;
    }
    __syncthreads();
    const int64_t t = s_task;
    if (t >= n_bt) break;
    const int64_t v = bt[4 * t], part = bt[4 * t + 1], k0 = bt[4 * t + 2], k1 = bt[4 * t + 3];
    const int64_t r0 = off[v] + part * kBlockDmax;
    const int64_t r1 = min(off[v + 1], r0 + kBlockDmax);
    Members m;
    m.words = bwords;
    m.cnt = bcnt;
    const int nclear = members_layout<PV>(m, col, r0, r1, kBlockWords, a.bitmap_bits);
    for (int i = tid; i < nclear; i += kThreads) {
      bwords[i] = m.bitmap ? 0 : kEmpty;
      if (PV) bcnt[i] = 0;
    }
    __syncthreads();
    for (int64_t p = r0 + tid; p < r1; p += kThreads) members_insert(m, col[p]);
    __syncthreads();
    // batches small enough that every warp gets several of them
    int64_t bsz = (k1 - k0) / (4 * kWarps);
    bsz = bsz < 1 ? 1 : (bsz > 32 ? 32 : bsz);
    int64_t h = stream_suffixes<PV>(rec, col, k0, k1, int(bsz), &s_batch, m, &s_bv[warp], pv, lane);
    acc += h;
    if (a.group) credit_group(a, v, h, lane);
    if (PV) {
      for (int o = 16; o; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
      if (lane == 0) s_red[warp] = (unsigned long long)h;
    }
    __syncthreads();
    if (PV) {
      if (tid == 0) {
        unsigned long long tot = 0;
        for (int w = 0; w < kWarps; w++) tot += s_red[w];
        if (tot) atomicAdd(reinterpret_cast<unsigned long long *>(&pv[v]), tot);
      }
      for (int i = tid; i < nclear; i += kThreads)
        if (bcnt[i]) atomicAdd(reinterpret_cast<unsigned long long *>(&pv[bwords[i]]), (unsigned long long)bcnt[i]);
      __syncthreads();
    }
  }

  // ---- warp tasks ----
  int32_t *wwords = wwords_all + warp * kWarpWords;
  int32_t *wcnt = wcnt_all + warp * kWarpWords;
  while (true) {
    int64_t t = 0;
    if (lane == 0) t = int64_t(atomicAdd(&cursor[1], 1ull));
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= n_wt) break;
    const int32_t v = wt[t];
    const int64_t r0 = off[v], r1 = off[v + 1];
    Members m;
    m.words = wwords;
    m.cnt = wcnt;
    const int nclear = members_layout<PV>(m, col, r0, r1, kWarpWords, a.bitmap_bits);
    for (int i = lane; i < nclear; i += 32) {
      wwords[i] = m.bitmap ? 0 : kEmpty;
      if (PV) wcnt[i] = 0;
    }
    __syncwarp();
    for (int64_t p = r0 + lane; p < r1; p += 32) members_insert(m, col[p]);
    __syncwarp();
    int64_t h = stream_suffixes<PV>(rec, col, ioff[v], ioff[v + 1], 32, nullptr, m, &s_bv[warp], pv, lane);
    acc += h;
    if (a.group) credit_group(a, v, h, lane);
    if (PV) {
      for (int o = 16; o; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
      __syncwarp();
      if (lane == 0 && h) atomicAdd(reinterpret_cast<unsigned long long *>(&pv[v]), (unsigned long long)h);
      for (int i = lane; i < nclear; i += 32)
        if (wcnt[i]) atomicAdd(reinterpret_cast<unsigned long long *>(&pv[wwords[i]]), (unsigned long long)wcnt[i]);
    }
    __syncwarp();
  }

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

static size_t count_smem_bytes(bool pv) {
  return sizeof(int32_t) * size_t(pv ? 2 : 1) * (kBlockWords + kWarps * kWarpWords);
}

// per-vertex counts in internal numbering -> input numbering
__global__ void k_unpermute(const int64_t *__restrict__ in, const int32_t *__restrict__ n2o, int64_t nv,
                            int64_t *__restrict__ out) {
  XT_GRID_STRIDE(r, nv) out[n2o[r]] = in[r];
}

__global__ void k_max_i32(const int32_t *__restrict__ a, int64_t n, unsigned long long *out) {
  unsigned long long m = 0;
  XT_GRID_STRIDE(i, n) m = max(m, (unsigned long long)a[i]);
  for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

__global__ void k_max_rowlen(const int64_t *__restrict__ off, int64_t nv, unsigned long long *out) {
  unsigned long long m = 0;
  XT_GRID_STRIDE(i, nv) m = max(m, (unsigned long long)(off[i + 1] - off[i]));
  for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
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
  dfree(c, g->plan->d_wt);
  dfree(c, g->plan->d_cursor);
  delete g->plan;
  g->plan = nullptr;
}

static xt_status d2h(Ctx *c, void *h, const void *d, size_t bytes) {
  return cuda_status(c, cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, c->stream), "D2H");
}

xt_status make_plan(Graph *g) {
  Ctx *c = g->ctx;
  free_plan(g);
  Plan *pl = new Plan();
  g->plan = pl;
  const int64_t nv = g->nv, ne = g->ne;
  const int B = 256;
  int64_t *w = nullptr, *P = nullptr, *nb = nullptr, *nw = nullptr, *nbp = nullptr, *nwp = nullptr;
  unsigned long long *stats = nullptr;
  xt_status s = XT_OK;
  do {
    if ((s = dalloc_n(c, &pl->d_cursor, 2)) != XT_OK) break;
    if ((s = dalloc_n(c, &stats, 4)) != XT_OK) break;
    if ((s = dalloc_n(c, &w, size_t(ne + 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &P, size_t(ne + 1))) != XT_OK) break;
    if ((s = cuda_status(c, cudaMemsetAsync(stats, 0, 4 * sizeof(unsigned long long), c->stream), "memset")) !=
        XT_OK)
      break;
    k_max_i32<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(g->d_deg, nv, stats + 0);
    k_max_rowlen<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(g->d_off, nv, stats + 1);
    k_max_rowlen<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(g->d_ioff, nv, stats + 2);
    // tail-grouped work, for the statistics only
    k_outedge_work<<<counted(c, grid_for(ne, B, c->sm_count)), B, 0, c->stream>>>(g->d_col, ne, g->d_off, w);
    if ((s = cuda_status(c, cudaMemsetAsync(w + ne, 0, sizeof(int64_t), c->stream), "memset")) != XT_OK) break;
    if ((s = exclusive_scan(c, w, P, ne + 1)) != XT_OK) break;
    int64_t tail_work = 0;
    if ((s = d2h(c, &tail_work, P + ne, sizeof(int64_t))) != XT_OK) break;
    // suffix lengths, prefix-summed in head order
    k_inrec_work<<<counted(c, grid_for(ne, B, c->sm_count)), B, 0, c->stream>>>(g->d_irec, ne, w);
    if ((s = exclusive_scan(c, w, P, ne + 1)) != XT_OK) break;
    // persistent grids: every CTA that fits on the device at once
    int occ[2] = {0, 0};
    for (int pvm = 0; pvm < 2 && s == XT_OK; pvm++) {
      auto fn = pvm ? k_count<true> : k_count<false>;
      const size_t bytes = count_smem_bytes(pvm != 0);
      s = cuda_status(c, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)), "attr");
      if (s == XT_OK)
        s = cuda_status(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[pvm], fn, kThreads, bytes), "occ");
    }
    if (s != XT_OK) break;
    pl->grid_global = c->sm_count * (occ[0] > 0 ? occ[0] : 1);
    pl->grid_pv = c->sm_count * (occ[1] > 0 ? occ[1] : 1);
    // CTA task size: large tasks amortise the member-set build and the task
    // barrier, but every CTA should still get about 16 of them
    int64_t total_work = 0;
    if ((s = d2h(c, &total_work, P + ne, sizeof(int64_t))) != XT_OK) break;
    if ((s = cuda_status(c, cudaStreamSynchronize(c->stream), "sync")) != XT_OK) break;
    PlanParams pp;
    pp.warp_dmax = kWarpDmax;
    pp.warp_work = g->tune_warp_work > 0 ? g->tune_warp_work : kWarpWork;
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
    k_plan_count<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(nv, g->d_off, g->d_ioff, P, pp, nb,
                                                                                nw);
    if ((s = cuda_status(c, cudaMemsetAsync(nb + nv, 0, sizeof(int64_t), c->stream), "memset")) != XT_OK) break;
    if ((s = cuda_status(c, cudaMemsetAsync(nw + nv, 0, sizeof(int64_t), c->stream), "memset")) != XT_OK) break;
    if ((s = exclusive_scan(c, nb, nbp, nv + 1)) != XT_OK) break;
    if ((s = exclusive_scan(c, nw, nwp, nv + 1)) != XT_OK) break;
    int64_t h[3] = {0, 0, 0};
    unsigned long long hs[4] = {0, 0, 0, 0};
    if ((s = d2h(c, &h[0], nbp + nv, sizeof(int64_t))) != XT_OK) break;
    if ((s = d2h(c, &h[1], nwp + nv, sizeof(int64_t))) != XT_OK) break;
    if ((s = d2h(c, &h[2], P + ne, sizeof(int64_t))) != XT_OK) break;
    if ((s = d2h(c, hs, stats, sizeof(hs))) != XT_OK) break;
    if ((s = cuda_status(c, cudaStreamSynchronize(c->stream), "sync")) != XT_OK) break;
    pl->n_btask = h[0];
    pl->n_wtask = h[1];
    g->max_degree = int64_t(hs[0]);
    g->max_out_degree = int64_t(hs[1]);
    g->max_in_degree = int64_t(hs[2]);
    g->wedge_work = tail_work;
    g->stream_work = h[2];
    if (g->max_out_degree >= kMaxOutDegree) {
      s = set_error(c, XT_ERR_OVERFLOW, "an oriented out-degree of 2^27 or more is not supported");
      break;
    }
    if ((s = dalloc_n(c, &pl->d_bt, size_t(4 * (pl->n_btask > 0 ? pl->n_btask : 1)))) != XT_OK) break;
    if ((s = dalloc_n(c, &pl->d_wt, size_t(pl->n_wtask > 0 ? pl->n_wtask : 1))) != XT_OK) break;
    k_plan_fill<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(nv, g->d_off, g->d_ioff, P, pp, nbp,
                                                                               nwp, pl->d_bt, pl->d_wt);
    if ((s = cuda_status(c, cudaGetLastError(), "k_plan_fill")) != XT_OK) break;
  } while (0);
  dfree(c, w);
  dfree(c, P);
  dfree(c, nb);
  dfree(c, nw);
  dfree(c, nbp);
  dfree(c, nwp);
  dfree(c, stats);
  if (s != XT_OK) free_plan(g);
  return s;
}

xt_status count_graph(Graph *g, int64_t *d_global, int64_t *d_pv, int64_t *d_groups) {
  Ctx *c = g->ctx;
  if (!g->plan) XT_TRY(make_plan(g));
  Plan *pl = g->plan;
  XT_CUDA(c, cudaMemsetAsync(pl->d_cursor, 0, 2 * sizeof(unsigned long long), c->stream));
  XT_CUDA(c, cudaMemsetAsync(d_global, 0, sizeof(int64_t), c->stream));
  if (d_groups) {
    if (!g->d_group) return set_error(c, XT_ERR_INVALID, "per-group counts need a graph built as a batch");
    XT_CUDA(c, cudaMemsetAsync(d_groups, 0, sizeof(int64_t) * g->n_groups, c->stream));
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
  a.ioff = g->d_ioff;
  a.rec = g->d_irec;
  a.bt = pl->d_bt;
  a.n_bt = pl->n_btask;
  a.wt = pl->d_wt;
  a.n_wt = pl->n_wtask;
  a.cursor = pl->d_cursor;
  a.global = reinterpret_cast<unsigned long long *>(d_global);
  a.pv = pv_int;
  a.group = d_groups ? g->d_group : nullptr;
  a.group_out = reinterpret_cast<unsigned long long *>(d_groups);
  a.bitmap_bits = pl->bitmap_bits;
  if (g->ne > 0) {
    if (d_pv)
      k_count<true><<<counted(c, pl->grid_pv), kThreads, count_smem_bytes(true), c->stream>>>(a);
    else
      k_count<false><<<counted(c, pl->grid_global), kThreads, count_smem_bytes(false), c->stream>>>(a);
  }
  if (d_pv && g->d_perm)
    k_unpermute<<<counted(c, grid_for(g->nv, 256, c->sm_count)), 256, 0, c->stream>>>(pv_int, g->d_perm, g->nv, d_pv);
  cudaError_t e = cudaGetLastError();
  if (pv_int && pv_int != d_pv) dfree(c, pv_int);
  XT_CUDA(c, e);
  return XT_OK;
}

}  // namespace xt
