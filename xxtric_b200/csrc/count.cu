// Degree-binned schedule and the exact triangle-count kernels.
//
// Orientation sends every undirected edge from its lower- to its higher-rank
// end, so every triangle {u,v,w} with rank u < v < w appears exactly once as
// u->v, u->w, v->w. The reference finds it from the lowest corner with a
// binary search per wedge (xxtric.hpp:150-207, counting.cu:579-638). Here it
// is found from the MIDDLE corner v: the out-list N+(v) is hashed once into
// shared memory, and the out-lists N+(u) of v's in-neighbours u are streamed
// through the hash; each hit w closes the triangle (u,v,w). The items read
// are sum_u d+(u)^2 instead of the tail-grouped sum over edges of d+(v),
// and every probe is a shared-memory lookup.
//
// Schedule (make_plan): per head v, work(v) = sum over u in N-(v) of d+(u).
//   warp bin : d+(v) <= kWarpDmax and work(v) <= kWarpWork -> one warp per v
//   block bin: d+(v) <= kBlockDmax -> CTA tasks over chunks of N-(v) of
//              about kBlockWork items each
//   part bin : d+(v) >  kBlockDmax -> N+(v) split into hash parts of
//              kBlockDmax keys, each part x each chunk one CTA task
// One persistent kernel drains the CTA tasks first (largest unit of work),
// then the warp tasks, each from a global atomic cursor.
#include <cub/cub.cuh>

#include "xt_internal.cuh"

namespace xt {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kWarpDmax = 64;     // warp hash: 128 slots
constexpr int kWarpSlots = 128;
constexpr int64_t kWarpWork = 2048;
constexpr int kBlockDmax = 2048;  // CTA hash: up to 4096 slots
constexpr int kBlockSlots = 4096;
constexpr int64_t kBlockWork = 1 << 16;
constexpr int32_t kEmpty = -1;

struct Plan {
  int64_t n_btask = 0;        // CTA tasks
  int64_t *d_bt = nullptr;    // 4 int64 per task: v, part, k0, k1 (k = index into d_icol)
  int64_t n_wtask = 0;        // warp tasks
  int32_t *d_wt = nullptr;    // v per warp task
  unsigned long long *d_cursor = nullptr;  // [0] CTA cursor, [1] warp cursor
  int grid = 0;
};

static unsigned grid_for(int64_t n, int block, int sm_count) {
  int64_t g = (n + block - 1) / block;
  int64_t cap = int64_t(sm_count) * 32;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (unsigned)g;
}

// ---- plan kernels -----------------------------------------------------------

// w[e] = d+(icol[e]) for every in-edge e (the items that edge streams)
__global__ void k_inedge_work(const int32_t *__restrict__ icol, int64_t ne, const int64_t *__restrict__ off,
                              int64_t *__restrict__ w) {
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < ne; e += int64_t(gridDim.x) * blockDim.x) {
    int32_t u = icol[e];
    w[e] = off[u + 1] - off[u];
  }
}

// tail-grouped work: d+(col[e]) per out-edge
__global__ void k_outedge_work(const int32_t *__restrict__ col, int64_t ne, const int64_t *__restrict__ off,
                               int64_t *__restrict__ w) {
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < ne; e += int64_t(gridDim.x) * blockDim.x) {
    int32_t v = col[e];
    w[e] = off[v + 1] - off[v];
  }
}

struct BinCounts {
  int64_t btasks;
  int64_t wtasks;
};

__device__ __forceinline__ void classify(int64_t v, const int64_t *__restrict__ off, const int64_t *__restrict__ ioff,
                                         const int64_t *__restrict__ P, int64_t &nb, int64_t &nw, int64_t &parts,
                                         int64_t &chunks, int64_t &work) {
  int64_t dp = off[v + 1] - off[v];
  int64_t k0 = ioff[v], k1 = ioff[v + 1];
  nb = nw = parts = chunks = 0;
  work = P[k1] - P[k0];
  if (dp == 0 || k1 == k0 || work == 0) return;
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
  for (int64_t v = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; v < nv; v += int64_t(gridDim.x) * blockDim.x) {
    int64_t nb, nw, parts, chunks, work;
    classify(v, off, ioff, P, nb, nw, parts, chunks, work);
    nb_out[v] = nb;
    nw_out[v] = nw;
  }
}

// first k in [lo,hi] with P[k] >= x
__device__ __forceinline__ int64_t lower_bound_i64(const int64_t *__restrict__ P, int64_t lo, int64_t hi, int64_t x) {
  while (lo < hi) {
    int64_t mid = lo + (hi - lo) / 2;
    if (P[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__global__ void k_plan_fill(int64_t nv, const int64_t *__restrict__ off, const int64_t *__restrict__ ioff,
                            const int64_t *__restrict__ P, const int64_t *__restrict__ nb_pos,
                            const int64_t *__restrict__ nw_pos, int64_t *__restrict__ bt, int32_t *__restrict__ wt) {
  for (int64_t v = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; v < nv; v += int64_t(gridDim.x) * blockDim.x) {
    int64_t nb, nw, parts, chunks, work;
    classify(v, off, ioff, P, nb, nw, parts, chunks, work);
    if (nw) wt[nw_pos[v]] = int32_t(v);
    if (!nb) continue;
    const int64_t k0 = ioff[v], k1 = ioff[v + 1], base = P[k0];
    int64_t t = nb_pos[v];
    int64_t prev = k0;
    for (int64_t c = 0; c < chunks; c++) {
      int64_t kend = (c + 1 == chunks) ? k1 : lower_bound_i64(P, prev, k1, base + (work * (c + 1)) / chunks);
      if (kend <= prev) continue;  // empty chunk (a single in-neighbour carries more work)
      for (int64_t p = 0; p < parts; p++) {
        bt[4 * t + 0] = v;
        bt[4 * t + 1] = p;
        bt[4 * t + 2] = prev;
        bt[4 * t + 3] = kend;
        t++;
      }
      prev = kend;
    }
    // unused slots (empty chunks) become no-op tasks
    for (; t < nb_pos[v] + nb; t++) {
      bt[4 * t + 0] = v;
      bt[4 * t + 1] = 0;
      bt[4 * t + 2] = k1;
      bt[4 * t + 3] = k1;
    }
  }
}

// ---- count kernel -----------------------------------------------------------

__device__ __forceinline__ uint32_t hash_slot(int32_t x, int shift) {
  return (uint32_t(x) * 0x9E3779B1u) >> shift;
}

template <bool PV>
__device__ __forceinline__ void hash_insert(int32_t *tab, uint32_t mask, int shift, int32_t x) {
  uint32_t h = hash_slot(x, shift);
  while (true) {
    int32_t old = atomicCAS(&tab[h], kEmpty, x);
    if (old == kEmpty || old == x) return;
    h = (h + 1) & mask;
  }
}

// returns the slot holding x, or -1
__device__ __forceinline__ int hash_find(const int32_t *tab, uint32_t mask, int shift, int32_t x) {
  uint32_t h = hash_slot(x, shift);
  while (true) {
    int32_t k = tab[h];
    if (k == x) return int(h);
    if (k == kEmpty) return -1;
    h = (h + 1) & mask;
  }
}

__device__ __forceinline__ int log2_slots(int64_t d, int min_slots) {
  int lg = 0;
  while ((int64_t(1) << lg) < 2 * d || (1 << lg) < min_slots) lg++;
  return lg;
}

// One warp streams the out-lists of in-neighbours icol[k] (k = kbeg, kbeg+kstep, ...
// in 32-wide batches) through the hash tab. Returns this lane's hit count.
template <bool PV>
__device__ __forceinline__ int64_t stream_inlists(const int64_t *__restrict__ off, const int32_t *__restrict__ col,
                                                  const int32_t *__restrict__ icol, int64_t kbeg, int64_t kend,
                                                  int64_t kstep, const int32_t *tab, int32_t *cnt, uint32_t mask,
                                                  int shift, int64_t *__restrict__ pv, int lane) {
  int64_t hits = 0;
  for (int64_t kb = kbeg; kb < kend; kb += kstep) {
    const int64_t k = kb + lane;
    int32_t u = 0;
    int64_t s = 0, e = 0;
    if (k < kend) {
      u = icol[k];
      s = off[u];
      e = off[u + 1];
    }
    const int nb = (kend - kb < 32) ? int(kend - kb) : 32;
    for (int j = 0; j < nb; j++) {
      const int64_t sj = __shfl_sync(0xffffffffu, s, j);
      const int64_t ej = __shfl_sync(0xffffffffu, e, j);
      int64_t h = 0;
      for (int64_t p = sj + lane; p < ej; p += 32) {
        const int32_t w = col[p];
        const int slot = hash_find(tab, mask, shift, w);
        if (slot >= 0) {
          h++;
          if (PV) atomicAdd(&cnt[slot], 1);
        }
      }
      hits += h;
      if (PV) {
        int64_t tot = h;
        for (int o = 16; o; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
        const int32_t uj = __shfl_sync(0xffffffffu, u, j);
        if (lane == 0 && tot) atomicAdd(reinterpret_cast<unsigned long long *>(&pv[uj]), (unsigned long long)tot);
      }
    }
  }
  return hits;
}

template <bool PV>
__global__ void __launch_bounds__(kThreads) k_count(const int64_t *__restrict__ off, const int32_t *__restrict__ col,
                                                    const int64_t *__restrict__ ioff,
                                                    const int32_t *__restrict__ icol, const int64_t *__restrict__ bt,
                                                    int64_t n_bt, const int32_t *__restrict__ wt, int64_t n_wt,
                                                    unsigned long long *__restrict__ cursor,
                                                    unsigned long long *__restrict__ global,
                                                    int64_t *__restrict__ pv) {
  extern __shared__ int32_t smem[];
  int32_t *btab = smem;                                       // kBlockSlots
  int32_t *bcnt = smem + kBlockSlots;                         // kBlockSlots (PV only)
  int32_t *wtab_all = smem + (PV ? 2 : 1) * kBlockSlots;      // kWarps * kWarpSlots
  int32_t *wcnt_all = wtab_all + kWarps * kWarpSlots;         // (PV only)
  __shared__ int64_t s_task;
  __shared__ unsigned long long s_red[kWarps];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int64_t acc = 0;

  // ---- CTA tasks ----
  while (true) {
    if (tid == 0) s_task = (int64_t)atomicAdd(&cursor[0], 1ull);
    __syncthreads();
    const int64_t t = s_task;
    if (t >= n_bt) break;
    const int64_t v = bt[4 * t], part = bt[4 * t + 1], k0 = bt[4 * t + 2], k1 = bt[4 * t + 3];
    const int64_t r0 = off[v] + part * kBlockDmax;
    const int64_t r1 = min(off[v + 1], r0 + kBlockDmax);
    const int lg = log2_slots(r1 - r0, 64);
    const uint32_t mask = (1u << lg) - 1;
    const int shift = 32 - lg;
    for (int i = tid; i <= int(mask); i += kThreads) {
      btab[i] = kEmpty;
      if (PV) bcnt[i] = 0;
    }
    __syncthreads();
    for (int64_t p = r0 + tid; p < r1; p += kThreads) hash_insert<PV>(btab, mask, shift, col[p]);
    __syncthreads();
    int64_t h = stream_inlists<PV>(off, col, icol, k0 + 32 * warp, k1, 32 * kWarps, btab, bcnt, mask, shift, pv, lane);
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
      for (int i = tid; i <= int(mask); i += kThreads)
        if (bcnt[i]) atomicAdd(reinterpret_cast<unsigned long long *>(&pv[btab[i]]), (unsigned long long)bcnt[i]);
      __syncthreads();
    }
  }

  // ---- warp tasks ----
  int32_t *wtab = wtab_all + warp * kWarpSlots;
  int32_t *wcnt = wcnt_all + warp * kWarpSlots;
  while (true) {
    int64_t t = 0;
    if (lane == 0) t = (int64_t)atomicAdd(&cursor[1], 1ull);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= n_wt) break;
    const int32_t v = wt[t];
    const int64_t r0 = off[v], r1 = off[v + 1];
    const int lg = log2_slots(r1 - r0, kWarpSlots);
    const uint32_t mask = (1u << lg) - 1;
    const int shift = 32 - lg;
    for (int i = lane; i < kWarpSlots; i += 32) {
      wtab[i] = kEmpty;
      if (PV) wcnt[i] = 0;
    }
    __syncwarp();
    for (int64_t p = r0 + lane; p < r1; p += 32) hash_insert<PV>(wtab, mask, shift, col[p]);
    __syncwarp();
    int64_t h = stream_inlists<PV>(off, col, icol, ioff[v], ioff[v + 1], 32, wtab, wcnt, mask, shift, pv, lane);
    acc += h;
    if (PV) {
      for (int o = 16; o; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
      __syncwarp();
      if (lane == 0 && h) atomicAdd(reinterpret_cast<unsigned long long *>(&pv[v]), (unsigned long long)h);
      for (int i = lane; i < kWarpSlots; i += 32)
        if (wcnt[i]) atomicAdd(reinterpret_cast<unsigned long long *>(&pv[wtab[i]]), (unsigned long long)wcnt[i]);
      __syncwarp();
    }
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
  return sizeof(int32_t) * ((pv ? 2 : 1) * kBlockSlots + (pv ? 2 : 1) * kWarps * kWarpSlots);
}

__global__ void k_max_i32(const int32_t *__restrict__ a, int64_t n, unsigned long long *out) {
  unsigned long long m = 0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    m = max(m, (unsigned long long)a[i]);
  for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

__global__ void k_max_rowlen(const int64_t *__restrict__ off, int64_t nv, unsigned long long *out) {
  unsigned long long m = 0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nv; i += int64_t(gridDim.x) * blockDim.x)
    m = max(m, (unsigned long long)(off[i + 1] - off[i]));
  for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// ---- host side --------------------------------------------------------------

template <class F>
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
    // graph statistics
    k_max_i32<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(g->d_deg, nv, stats + 0);
    k_max_rowlen<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(g->d_off, nv, stats + 1);
    k_max_rowlen<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(g->d_ioff, nv, stats + 2);
    // tail-grouped work (statistics only)
    k_outedge_work<<<counted(c, grid_for(ne, B, c->sm_count)), B, 0, c->stream>>>(g->d_col, ne, g->d_off, w);
    if ((s = cuda_status(c, cudaMemsetAsync(w + ne, 0, sizeof(int64_t), c->stream), "memset")) != XT_OK) break;
    if ((s = exclusive_scan<int64_t>(c, w, P, ne + 1)) != XT_OK) break;
    int64_t tail_work = 0;
    if ((s = cuda_status(c, cudaMemcpyAsync(&tail_work, P + ne, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream),
                         "memcpy")) != XT_OK)
      break;
    // head-grouped work prefix over in-edges
    k_inedge_work<<<counted(c, grid_for(ne, B, c->sm_count)), B, 0, c->stream>>>(g->d_icol, ne, g->d_off, w);
    if ((s = exclusive_scan<int64_t>(c, w, P, ne + 1)) != XT_OK) break;
    if ((s = dalloc_n(c, &nb, size_t(nv + 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &nw, size_t(nv + 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &nbp, size_t(nv + 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &nwp, size_t(nv + 1))) != XT_OK) break;
    k_plan_count<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(nv, g->d_off, g->d_ioff, P, nb, nw);
    if ((s = cuda_status(c, cudaMemsetAsync(nb + nv, 0, sizeof(int64_t), c->stream), "memset")) != XT_OK) break;
    if ((s = cuda_status(c, cudaMemsetAsync(nw + nv, 0, sizeof(int64_t), c->stream), "memset")) != XT_OK) break;
    if ((s = exclusive_scan<int64_t>(c, nb, nbp, nv + 1)) != XT_OK) break;
    if ((s = exclusive_scan<int64_t>(c, nw, nwp, nv + 1)) != XT_OK) break;
    int64_t h[2] = {0, 0};
    unsigned long long hs[4] = {0, 0, 0, 0};
    if ((s = cuda_status(c, cudaMemcpyAsync(&h[0], nbp + nv, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream),
                         "memcpy")) != XT_OK)
      break;
    if ((s = cuda_status(c, cudaMemcpyAsync(&h[1], nwp + nv, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream),
                         "memcpy")) != XT_OK)
      break;
    int64_t head_work = 0;
    if ((s = cuda_status(c, cudaMemcpyAsync(&head_work, P + ne, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream),
                         "memcpy")) != XT_OK)
      break;
    if ((s = cuda_status(c, cudaMemcpyAsync(hs, stats, sizeof(hs), cudaMemcpyDeviceToHost, c->stream), "memcpy")) !=
        XT_OK)
      break;
    if ((s = cuda_status(c, cudaStreamSynchronize(c->stream), "sync")) != XT_OK) break;
    pl->n_btask = h[0];
    pl->n_wtask = h[1];
    g->max_degree = int64_t(hs[0]);
    g->max_out_degree = int64_t(hs[1]);
    g->max_in_degree = int64_t(hs[2]);
    g->wedge_work = tail_work;
    g->stream_work = head_work;
    if ((s = dalloc_n(c, &pl->d_bt, size_t(4 * (pl->n_btask > 0 ? pl->n_btask : 1)))) != XT_OK) break;
    if ((s = dalloc_n(c, &pl->d_wt, size_t(pl->n_wtask > 0 ? pl->n_wtask : 1))) != XT_OK) break;
    k_plan_fill<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(nv, g->d_off, g->d_ioff, P, nbp, nwp, pl->d_bt,
                                                                   pl->d_wt);
    if ((s = cuda_status(c, cudaGetLastError(), "k_plan_fill")) != XT_OK) break;
    // persistent grid
    const size_t sm_bytes = count_smem_bytes(true);
    if ((s = cuda_status(c, cudaFuncSetAttribute(k_count<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 int(sm_bytes)),
                         "attr")) != XT_OK)
      break;
    if ((s = cuda_status(c, cudaFuncSetAttribute(k_count<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 int(count_smem_bytes(false))),
                         "attr")) != XT_OK)
      break;
    int occ = 0;
    if ((s = cuda_status(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_count<false>, kThreads,
                                                                            count_smem_bytes(false)),
                         "occupancy")) != XT_OK)
      break;
    pl->grid = c->sm_count * (occ > 0 ? occ : 1);
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
  if (d_pv) XT_CUDA(c, cudaMemsetAsync(d_pv, 0, sizeof(int64_t) * g->nv, c->stream));
  if (g->ne == 0) return XT_OK;
  unsigned long long *gl = reinterpret_cast<unsigned long long *>(d_global);
  if (d_pv)
    k_count<true><<<counted(c, pl->grid), kThreads, count_smem_bytes(true), c->stream>>>(
        g->d_off, g->d_col, g->d_ioff, g->d_icol, pl->d_bt, pl->n_btask, pl->d_wt, pl->n_wtask, pl->d_cursor, gl,
        d_pv);
  else
    k_count<false><<<counted(c, pl->grid), kThreads, count_smem_bytes(false), c->stream>>>(
        g->d_off, g->d_col, g->d_ioff, g->d_icol, pl->d_bt, pl->n_btask, pl->d_wt, pl->n_wtask, pl->d_cursor, gl,
        nullptr);
  XT_CUDA(c, cudaGetLastError());
  return XT_OK;
}

}  // namespace xt
