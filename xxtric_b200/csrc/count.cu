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

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kWarpDmax = 64;
constexpr int kWarpWords = 256;   // per-warp region: 256-slot hash or 8192-bit bitmap
constexpr int64_t kWarpWork = 4096;
constexpr int kBlockDmax = 2048;
constexpr int kBlockWords = 8192;  // CTA region: 8192-slot hash or 2^18-bit bitmap
constexpr int64_t kBlockWork = 1 << 18;
constexpr int32_t kEmpty = -1;

struct Plan {
  int64_t n_btask = 0;        // CTA tasks
  int64_t *d_bt = nullptr;    // 4 int64 per task: v, part, k0, k1 (k = in-record index)
  int64_t n_wtask = 0;        // warp tasks
  int32_t *d_wt = nullptr;    // v per warp task
  unsigned long long *d_cursor = nullptr;  // [0] CTA cursor, [1] warp cursor
  int grid_global = 0, grid_pv = 0;
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
                                         const int64_t *__restrict__ P, int64_t &nb, int64_t &nw, int64_t &parts,
                                         int64_t &chunks, int64_t &work) {
  const int64_t dp = off[v + 1] - off[v];
  const int64_t k0 = ioff[v], k1 = ioff[v + 1];
  nb = nw = parts = chunks = 0;
  work = P[k1] - P[k0];
  if (dp == 0 || work == 0) return;
  if (dp <= kWarpDmax && work <= kWarpWork) {
    nw = 1;
    return;
  }
  parts = (dp + kBlockDmax - 1) / kBlockDmax;
  chunks = (work + kBlockWork - 1) / kBlockWork;
  nb = parts * chunks;
}

__global__ void k_plan_count(int64_t nv, const int64_t *__restrict__ off, const int64_t *__restrict__ ioff,
                             const int64_t *__restrict__ P, int64_t *__restrict__ nb_out,
                             int64_t *__restrict__ nw_out) {
  XT_GRID_STRIDE(v, nv) {
    int64_t nb, nw, parts, chunks, work;
    classify(v, off, ioff, P, nb, nw, parts, chunks, work);
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
                            const int64_t *__restrict__ P, const int64_t *__restrict__ nb_pos,
                            const int64_t *__restrict__ nw_pos, int64_t *__restrict__ bt, int32_t *__restrict__ wt) {
  XT_GRID_STRIDE(v, nv) {
    int64_t nb, nw, parts, chunks, work;
    classify(v, off, ioff, P, nb, nw, parts, chunks, work);
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

// Chooses the structure for members col[r0, r1) that fits `words` words and
// returns how many words must be cleared.
template <bool PV>
__device__ __forceinline__ int members_layout(Members &m, const int32_t *__restrict__ col, int64_t r0, int64_t r1,
                                              int words) {
  m.lo = col[r0];
  m.hi = col[r1 - 1];
  const int64_t range = int64_t(m.hi) - int64_t(m.lo) + 1;
  m.bitmap = !PV && range <= int64_t(words) * 32;
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

// A warp step: 32 aligned 16-byte groups (one LDG.128 per lane) of one suffix.
struct Chunk {
  int4 x;          // four columns of this lane's group
  int64_t grp;     // group index (columns 4*grp .. 4*grp+3)
  int64_t s, e;    // the suffix [s, e)
  int32_t u;       // its owner (per-vertex credit)
  int32_t serial;  // which suffix of the walk (warp-uniform)
  bool exists;     // warp-uniform: this step exists
};

// One warp's walk over the in-records rec[k0, kend), taken in batches of bsz
// records (lane j < bsz holds record j of a batch). Batches come one after
// another (a warp task), or from a cursor in shared memory that the warps of
// a CTA task share, so warps that finish early take more. The next batch is
// claimed and its records loaded while the current one streams.
// Control flow is warp-uniform.
struct RecWalk {
  const InRec *__restrict__ rec;
  const int32_t *__restrict__ col;
  int *cursor;              // shared batch cursor (CTA task) or null
  int64_t k0, kend;         // the task's records
  int64_t kb, nkb, seq;     // current / next batch base, next sequential base
  int bsz, nb, j;
  int64_t bs, be;           // lane's record of this batch
  int32_t bu;
  int4 nrec;                // lane's record of the next batch (prefetched)
  int64_t cs, ce, g, gend;  // current suffix and group cursor
  int32_t cu, serial;
  bool have;
  int lane;

  __device__ __forceinline__ int64_t claim() {
    if (!cursor) {
      const int64_t b = seq;
      seq += bsz;
      return b;
    }
    int r = 0;
    if (lane == 0) r = atomicAdd(cursor, bsz);
    return k0 + __shfl_sync(0xffffffffu, r, 0);
  }
  __device__ __forceinline__ int4 fetch(int64_t base) const {
    const int64_t k = base + lane;
    return (lane < bsz && k < kend) ? __ldg(reinterpret_cast<const int4 *>(rec) + k) : make_int4(0, 0, 0, -1);
  }
  __device__ __forceinline__ void take(int4 r) {
    bs = int64_t(uint32_t(r.x)) | (int64_t(r.y) << 32);
    be = bs + r.z;
    bu = r.w;
    nb = (kend - kb < bsz) ? int(kend - kb) : bsz;
    nkb = claim();
    nrec = fetch(nkb);
  }
  __device__ __forceinline__ void select(int jj) {
    j = jj;
    cs = __shfl_sync(0xffffffffu, bs, jj);
    ce = __shfl_sync(0xffffffffu, be, jj);
    cu = __shfl_sync(0xffffffffu, bu, jj);
    g = cs >> 2;
    gend = (ce + 3) >> 2;
    if (cs == ce) gend = g;  // empty suffix
    serial++;
  }
  __device__ __forceinline__ void init() {
    nb = j = 0;
    bs = be = cs = ce = g = gend = 0;
    bu = cu = -1;
    serial = 0;
    seq = k0;
    kb = claim();
    have = kb < kend;
    if (!have) return;
    take(fetch(kb));
    select(0);
  }
  __device__ __forceinline__ void advance() {
    while (have && g >= gend) {
      if (j + 1 < nb) {
        select(j + 1);
      } else {
        kb = nkb;
        if (kb >= kend) {
          have = false;
          break;
        }
        take(nrec);
        select(0);
      }
    }
  }
  __device__ __forceinline__ Chunk issue() {
    Chunk c;
    advance();
    c.exists = have;
    c.grp = g + lane;
    c.s = cs;
    c.e = ce;
    c.u = cu;
    c.serial = serial;
    c.x = make_int4(0, 0, 0, 0);
    if (have) {
      if (c.grp < gend) c.x = __ldg(reinterpret_cast<const int4 *>(col) + c.grp);
      g += 32;
    }
    return c;
  }
};

// Probes a chunk; returns this lane's hits and sets `past` when none of the
// lane's valid columns is <= m.hi (so the rest of the suffix is past it).
template <bool PV>
__device__ __forceinline__ int probe_chunk(const Chunk &c, const Members &m, bool &past) {
  int h = 0;
  past = true;
  const int64_t p0 = 4 * c.grp;
  const int32_t w[4] = {c.x.x, c.x.y, c.x.z, c.x.w};
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int64_t p = p0 + i;
    if (p < c.s || p >= c.e) continue;
    const int32_t x = w[i];
    if (x <= m.hi) past = false;
    if (x < m.lo || x > m.hi) continue;
    if (m.bitmap) {
      const uint32_t d = uint32_t(x - m.lo);
      h += (m.words[d >> 5] >> (d & 31)) & 1;
    } else {
      const int slot = hash_find(m.words, m.mask, m.shift, x);
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
template <bool PV>
__device__ __forceinline__ int64_t stream_suffixes(const InRec *__restrict__ rec, const int32_t *__restrict__ col,
                                                   int64_t k0, int64_t kend, int bsz, int *cursor, const Members &m,
                                                   int64_t *__restrict__ pv, int lane) {
  RecWalk wk;
  wk.rec = rec;
  wk.col = col;
  wk.cursor = cursor;
  wk.k0 = k0;
  wk.kend = kend;
  wk.bsz = bsz;
  wk.lane = lane;
  wk.init();
  int64_t hits = 0;
  Chunk a = wk.issue();
  while (a.exists) {
    Chunk b = wk.issue();  // the next step's loads are in flight during these probes
    bool past;
    const int h = probe_chunk<PV>(a, m, past);
    hits += h;
    if (PV) {
      int tot = h;
      for (int o = 16; o; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
      if (lane == 0 && tot) atomicAdd(reinterpret_cast<unsigned long long *>(&pv[a.u]), (unsigned long long)tot);
    }
    if (__all_sync(0xffffffffu, past) && b.exists && b.serial == a.serial) {
      // the suffix is sorted: every later column is above max N+(v) too, so
      // drop the step already in flight and the rest of this suffix
      wk.g = wk.gend;
      b = wk.issue();
    }
    a = b;
  }
  return hits;
}

// ---- the count kernel ---------------------------------------------------------

template <bool PV>
__global__ void __launch_bounds__(kThreads, 4) k_count(const int64_t *__restrict__ off, const int32_t *__restrict__ col,
                                                       const int64_t *__restrict__ ioff,
                                                       const InRec *__restrict__ rec, const int64_t *__restrict__ bt,
                                                       int64_t n_bt, const int32_t *__restrict__ wt, int64_t n_wt,
                                                       unsigned long long *__restrict__ cursor,
                                                       unsigned long long *__restrict__ global,
                                                       int64_t *__restrict__ pv) {
  extern __shared__ int32_t smem[];
  int32_t *bwords = smem;                                   // kBlockWords
  int32_t *bcnt = smem + kBlockWords;                       // kBlockWords (PV only)
  int32_t *wwords_all = smem + (PV ? 2 : 1) * kBlockWords;  // kWarps * kWarpWords
  int32_t *wcnt_all = wwords_all + kWarps * kWarpWords;     // (PV only)
  __shared__ int64_t s_task;
  __shared__ int s_batch;  // next in-record batch of the current CTA task
  __shared__ unsigned long long s_red[kWarps];

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
    const int nclear = members_layout<PV>(m, col, r0, r1, kBlockWords);
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
    int64_t h = stream_suffixes<PV>(rec, col, k0, k1, int(bsz), &s_batch, m, pv, lane);
    acc += h;
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
    const int nclear = members_layout<PV>(m, col, r0, r1, kWarpWords);
    for (int i = lane; i < nclear; i += 32) {
      wwords[i] = m.bitmap ? 0 : kEmpty;
      if (PV) wcnt[i] = 0;
    }
    __syncwarp();
    for (int64_t p = r0 + lane; p < r1; p += 32) members_insert(m, col[p]);
    __syncwarp();
    int64_t h = stream_suffixes<PV>(rec, col, ioff[v], ioff[v + 1], 32, nullptr, m, pv, lane);
    acc += h;
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
    atomicAdd(global, tot);
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
    if ((s = dalloc_n(c, &nb, size_t(nv + 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &nw, size_t(nv + 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &nbp, size_t(nv + 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &nwp, size_t(nv + 1))) != XT_OK) break;
    k_plan_count<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(nv, g->d_off, g->d_ioff, P, nb, nw);
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
    if ((s = dalloc_n(c, &pl->d_bt, size_t(4 * (pl->n_btask > 0 ? pl->n_btask : 1)))) != XT_OK) break;
    if ((s = dalloc_n(c, &pl->d_wt, size_t(pl->n_wtask > 0 ? pl->n_wtask : 1))) != XT_OK) break;
    k_plan_fill<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(nv, g->d_off, g->d_ioff, P, nbp, nwp,
                                                                               pl->d_bt, pl->d_wt);
    if ((s = cuda_status(c, cudaGetLastError(), "k_plan_fill")) != XT_OK) break;
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

xt_status count_graph(Graph *g, int64_t *d_global, int64_t *d_pv) {
  Ctx *c = g->ctx;
  if (!g->plan) XT_TRY(make_plan(g));
  Plan *pl = g->plan;
  XT_CUDA(c, cudaMemsetAsync(pl->d_cursor, 0, 2 * sizeof(unsigned long long), c->stream));
  XT_CUDA(c, cudaMemsetAsync(d_global, 0, sizeof(int64_t), c->stream));
  int64_t *pv_int = nullptr;  // per-vertex counts in internal numbering
  if (d_pv) {
    if (g->d_perm) XT_TRY(dalloc_n(c, &pv_int, size_t(g->nv)));
    else pv_int = d_pv;
    XT_CUDA(c, cudaMemsetAsync(pv_int, 0, sizeof(int64_t) * g->nv, c->stream));
  }
  unsigned long long *gl = reinterpret_cast<unsigned long long *>(d_global);
  if (g->ne > 0) {
    if (d_pv)
      k_count<true><<<counted(c, pl->grid_pv), kThreads, count_smem_bytes(true), c->stream>>>(
          g->d_off, g->d_col, g->d_ioff, g->d_irec, pl->d_bt, pl->n_btask, pl->d_wt, pl->n_wtask, pl->d_cursor, gl,
          pv_int);
    else
      k_count<false><<<counted(c, pl->grid_global), kThreads, count_smem_bytes(false), c->stream>>>(
          g->d_off, g->d_col, g->d_ioff, g->d_irec, pl->d_bt, pl->n_btask, pl->d_wt, pl->n_wtask, pl->d_cursor, gl,
          nullptr);
  }
  if (d_pv && g->d_perm)
    k_unpermute<<<counted(c, grid_for(g->nv, 256, c->sm_count)), 256, 0, c->stream>>>(pv_int, g->d_perm, g->nv, d_pv);
  cudaError_t e = cudaGetLastError();
  if (pv_int && pv_int != d_pv) dfree(c, pv_int);
  XT_CUDA(c, e);
  return XT_OK;
}

}  // namespace xt
