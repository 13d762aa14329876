// The batching form: many independent graphs counted in one launch. It has
// no counterpart in the reference, whose driver reads or generates one graph
// per run and counts it once (main.cpp:76-192); each graph's count here
// equals what the plain single-graph path returns for it.
//
// Layout: the graphs are one disjoint union. Graph g owns the ids
// [voff[g], voff[g+1]) of one concatenated CSR built by the ordinary builder
// (so one sort serves all graphs), and a per-vertex group map sends every
// task's hits to its graph's counter. Triangles never cross graphs, so the
// per-graph counts are exactly those of counting each graph alone; the plan
// (bins, tasks) and the persistent kernel are the plain ones, with a work
// queue over all graphs' (head, chunk) tiles.
//
// Also here: the batch workload's generators (per graph: an Erdos-Renyi or a
// unit-square random geometric graph with its own size and mean degree, all
// drawn from one seed), CUDA-graph capture of a count, and the autotuner.
#include <cub/cub.cuh>

#include <new>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "xt_internal.cuh"
#include "xt_rng.cuh"

namespace xt {

static unsigned grid_for(int64_t n, int block, int sm_count) {
  int64_t g = (n + block - 1) / block;
  int64_t cap = int64_t(sm_count) * 32;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (unsigned)g;
}

#define XT_GRID_STRIDE(i, n) \
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < (n); i += int64_t(gridDim.x) * blockDim.x)

constexpr uint64_t kStreamBatch = 5, kStreamRgg = 4, kStreamER = 3;

// largest i with off[i] <= x, for off[0] = 0 <= x < off[n]
__device__ __forceinline__ int64_t find_seg(const int64_t *__restrict__ off, int64_t n, int64_t x) {
  int64_t lo = 0, hi = n;
  while (hi - lo > 1) {
    const int64_t mid = lo + (hi - lo) / 2;
    if (off[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

// ---- union build ----------------------------------------------------------

__global__ void k_globalize(const int32_t *__restrict__ src, const int32_t *__restrict__ dst, int64_t ne,
                            const int64_t *__restrict__ eoff, const int64_t *__restrict__ voff, int64_t ng,
                            int32_t *__restrict__ gsrc, int32_t *__restrict__ gdst, int *__restrict__ err) {
  XT_GRID_STRIDE(e, ne) {
    const int64_t g = find_seg(eoff, ng, e);
    const int64_t n = voff[g + 1] - voff[g];
    int64_t s = src[e], d = dst[e];
    if (s < 0 || d < 0 || s >= n || d >= n) {
      atomicOr(err, 1);
      s = 0;
      d = 0;
    }
    gsrc[e] = int32_t(voff[g] + s);
    gdst[e] = int32_t(voff[g] + d);
  }
}

// internal id -> graph
__global__ void k_group_of(const int32_t *__restrict__ perm, int64_t nv, const int64_t *__restrict__ voff, int64_t ng,
                           int32_t *__restrict__ group) {
  XT_GRID_STRIDE(r, nv) {
    const int64_t input = perm ? perm[r] : r;
    group[r] = int32_t(find_seg(voff, ng, input));
  }
}

xt_status build_batch(Ctx *c, int64_t ng, const int64_t *h_voff, const int64_t *h_eoff, const int32_t *d_src,
                      const int32_t *d_dst, int orient, Graph *g) {
  if (ng < 1 || !h_voff || !h_eoff) return set_error(c, XT_ERR_INVALID, "batch: bad graph tables");
  if (h_voff[0] != 0 || h_eoff[0] != 0) return set_error(c, XT_ERR_INVALID, "batch: offsets must start at 0");
  for (int64_t i = 0; i < ng; i++)
    if (h_voff[i + 1] < h_voff[i] || h_eoff[i + 1] < h_eoff[i])
      return set_error(c, XT_ERR_INVALID, "batch: offsets must not decrease");
  const int64_t nv = h_voff[ng], ne = h_eoff[ng];
  if (nv < 1) return set_error(c, XT_ERR_INVALID, "batch: no vertices");
  if (nv > (int64_t(1) << 31) - 1) return set_error(c, XT_ERR_OVERFLOW, "batch: 2^31 or more vertices in all");
  int64_t *d_voff = nullptr, *d_eoff = nullptr;
  int32_t *gs = nullptr, *gd = nullptr;
  xt_status s = XT_OK;
  do {
    if ((s = dalloc_n(c, &d_voff, size_t(ng + 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &d_eoff, size_t(ng + 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &gs, size_t(ne > 0 ? ne : 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &gd, size_t(ne > 0 ? ne : 1))) != XT_OK) break;
    if ((s = cuda_status(c, cudaMemcpyAsync(d_voff, h_voff, sizeof(int64_t) * (ng + 1), cudaMemcpyHostToDevice,
                                            c->stream), "H2D")) != XT_OK)
      break;
    if ((s = cuda_status(c, cudaMemcpyAsync(d_eoff, h_eoff, sizeof(int64_t) * (ng + 1), cudaMemcpyHostToDevice,
                                            c->stream), "H2D")) != XT_OK)
      break;
    if (ne > 0)
      k_globalize<<<counted(c, grid_for(ne, 256, c->sm_count)), 256, 0, c->stream>>>(d_src, d_dst, ne, d_eoff, d_voff,
                                                                                     ng, gs, gd, c->d_err);
    int h = 0;
    if ((s = cuda_status(c, cudaMemcpyAsync(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "D2H")) !=
        XT_OK)
      break;
    if ((s = cuda_status(c, cudaStreamSynchronize(c->stream), "sync")) != XT_OK) break;
    if (h) {
      cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream);
      s = set_error(c, XT_ERR_INVALID, "batch: a vertex id is outside its graph");
      break;
    }
    if ((s = build_from_edges(c, nv, ne, gs, gd, orient, g)) != XT_OK) break;
    dfree(c, gs);
    dfree(c, gd);
    gs = gd = nullptr;
    if ((s = dalloc_n(c, &g->d_group, size_t(nv))) != XT_OK) break;
    k_group_of<<<counted(c, grid_for(nv, 256, c->sm_count)), 256, 0, c->stream>>>(g->d_perm, nv, d_voff, ng,
                                                                                   g->d_group);
    g->n_groups = ng;
    s = cuda_status(c, cudaGetLastError(), "k_group_of");
  } while (0);
  dfree(c, d_voff);
  dfree(c, d_eoff);
  dfree(c, gs);
  dfree(c, gd);
  return s;
}

// ---- the batch workload's generators ---------------------------------------

// Erdos-Renyi edges of every kind-1 graph: m pairs of local ids
__global__ void k_batch_er(int64_t ng, const int32_t *__restrict__ kind, const int64_t *__restrict__ nvtx,
                           const uint64_t *__restrict__ gseed, const int64_t *__restrict__ eoff, int64_t ne,
                           int32_t *__restrict__ src, int32_t *__restrict__ dst) {
  XT_GRID_STRIDE(e, ne) {
    const int64_t g = find_seg(eoff, ng, e);
    if (kind[g] != 1) continue;
    const uint64_t k = uint64_t(e - eoff[g]), n = uint64_t(nvtx[g]);
    src[e] = int32_t(__umul64hi(crand(gseed[g], kStreamER, 2u * k), n));
    dst[e] = int32_t(__umul64hi(crand(gseed[g], kStreamER, 2u * k + 1u), n));
  }
}

// unit-square points of the kind-0 graphs and their cell keys
__global__ void k_batch_points(int64_t ng, const int32_t *__restrict__ kind, const int64_t *__restrict__ poff,
                               const uint64_t *__restrict__ gseed, const int32_t *__restrict__ cells,
                               const int64_t *__restrict__ cbase, int64_t np, double *__restrict__ x,
                               double *__restrict__ y, uint32_t *__restrict__ key, int32_t *__restrict__ idx) {
  const double inv53 = 1.0 / 9007199254740992.0;  // 2^-53
  XT_GRID_STRIDE(p, np) {
    const int64_t g = find_seg(poff, ng, p);
    const uint64_t i = uint64_t(p - poff[g]);
    const double px = double(crand(gseed[g], kStreamRgg, 2u * i) >> 11) * inv53;
    const double py = double(crand(gseed[g], kStreamRgg, 2u * i + 1u) >> 11) * inv53;
    x[p] = px;
    y[p] = py;
    const int32_t C = cells[g];
    int32_t cx = int32_t(px * double(C)), cy = int32_t(py * double(C));
    cx = cx >= C ? C - 1 : cx;
    cy = cy >= C ? C - 1 : cy;
    key[p] = (kind[g] == 0) ? uint32_t(cbase[g] + int64_t(cy) * C + cx) : 0xffffffffu;
    idx[p] = int32_t(p);
  }
}

// sorted cell keys -> first point of every cell (cstart[ncell] = points with a cell)
__global__ void k_cell_starts(const uint32_t *__restrict__ skey, int64_t np, int64_t ncell,
                              int64_t *__restrict__ cstart) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i <= np; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t prev = (i == 0) ? -1 : (skey[i - 1] == 0xffffffffu ? ncell : int64_t(skey[i - 1]));
    const int64_t cur = (i == np || skey[i] == 0xffffffffu) ? ncell : int64_t(skey[i]);
    for (int64_t c = prev + 1; c <= cur && c <= ncell; c++) cstart[c] = i;
  }
}

// pairs u < v (local ids) of one kind-0 graph within distance sqrt(r2): pass 0
// counts per point, pass 1 writes at the scanned positions. The distance test
// uses explicit round-to-nearest products and sums (no fused multiply-add),
// the same IEEE expression the CPU evaluates.
template <bool WRITE>
__global__ void k_batch_rgg(int64_t ng, const int32_t *__restrict__ kind, const int64_t *__restrict__ poff,
                            const double *__restrict__ r2, const int32_t *__restrict__ cells,
                            const int64_t *__restrict__ cbase, const double *__restrict__ x,
                            const double *__restrict__ y, const int32_t *__restrict__ order,
                            const int64_t *__restrict__ cstart, int64_t np, int64_t *__restrict__ cnt,
                            const int64_t *__restrict__ pos, int32_t *__restrict__ src, int32_t *__restrict__ dst) {
  XT_GRID_STRIDE(p, np) {
    const int64_t g = find_seg(poff, ng, p);
    if (kind[g] != 0) {
      if (!WRITE) cnt[p] = 0;
      continue;
    }
    const int32_t C = cells[g];
    const double px = x[p], py = y[p], rr = r2[g];
    int32_t cx = int32_t(px * double(C)), cy = int32_t(py * double(C));
    cx = cx >= C ? C - 1 : cx;
    cy = cy >= C ? C - 1 : cy;
    int64_t k = 0;
    const int64_t w = WRITE ? pos[p] : 0;
    for (int dy = -1; dy <= 1; dy++)
      for (int dx = -1; dx <= 1; dx++) {
        const int32_t nx = cx + dx, ny = cy + dy;
        if (nx < 0 || ny < 0 || nx >= C || ny >= C) continue;
        const int64_t cell = cbase[g] + int64_t(ny) * C + nx;
        for (int64_t t = cstart[cell]; t < cstart[cell + 1]; t++) {
          const int64_t q = order[t];
          if (q <= p) continue;
          const double ddx = __dsub_rn(px, x[q]), ddy = __dsub_rn(py, y[q]);
          const double d2 = __dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy));
          if (d2 <= rr) {
            if (WRITE) {
              src[w + k] = int32_t(p - poff[g]);
              dst[w + k] = int32_t(q - poff[g]);
            }
            k++;
          }
        }
      }
    if (!WRITE) cnt[p] = k;
  }
}

static xt_status scan_i64(Ctx *c, const int64_t *in, int64_t *out, int64_t n) {
  size_t bytes = 0;
  XT_CUDA(c, cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, c->stream));
  void *tmp = nullptr;
  XT_TRY(dalloc(c, &tmp, bytes));
  cudaError_t e = cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, n, c->stream);
  dfree(c, tmp);
  XT_CUDA(c, e);
  return XT_OK;
}

// RGG cells per side for radius^2 r2: no smaller than the radius (every pair
// within it lies in the same or an adjacent cell), at most 4096
static int32_t rgg_cells(double r2) {
  double c = std::floor(1.0 / (std::sqrt(r2) * 1.0001));
  if (c < 1.0) c = 1.0;
  if (c > 4096.0) c = 4096.0;
  return int32_t(c);
}

// pos[p] += shift[graph of p]
__global__ void k_shift_pos(int64_t ng, const int64_t *__restrict__ poff, const int64_t *__restrict__ shift,
                            int64_t np, int64_t *__restrict__ pos) {
  XT_GRID_STRIDE(p, np) pos[p] += shift[find_seg(poff, ng, p)];
}

xt_status gen_batch(Ctx *c, int64_t ng, const int32_t *kind, const int64_t *nvtx, const double *deg,
                    const uint64_t *gseed, int64_t *h_eoff, int32_t **d_src_out, int32_t **d_dst_out) {
  // 1. host tables
  std::vector<int64_t> poff(ng + 1, 0), cbase(ng + 1, 0), m(ng, 0);
  std::vector<int32_t> cells(ng, 1);
  std::vector<double> r2(ng, 0.0);
  for (int64_t g = 0; g < ng; g++) {
    if (nvtx[g] < 1 || (kind[g] != 0 && kind[g] != 1) || !(deg[g] > 0)) return set_error(c, XT_ERR_INVALID, "batch spec");
    poff[g + 1] = poff[g] + nvtx[g];
    if (kind[g] == 0) {
      r2[g] = deg[g] / (3.14159265358979323846 * double(nvtx[g]));
      cells[g] = rgg_cells(r2[g]);
    } else {
      m[g] = int64_t(std::llround(double(nvtx[g]) * deg[g] / 2.0));
    }
    cbase[g + 1] = cbase[g] + (kind[g] == 0 ? int64_t(cells[g]) * cells[g] : 0);
  }
  const int64_t np = poff[ng], ncell = cbase[ng];
  if (ncell >= int64_t(0xffffffffu)) return set_error(c, XT_ERR_OVERFLOW, "batch: too many cells");
  const int B = 256;
  // device copies of the tables
  int32_t *d_kind = nullptr, *d_cells = nullptr, *d_order = nullptr, *d_idx = nullptr;
  int64_t *d_n = nullptr, *d_poff = nullptr, *d_cbase = nullptr, *d_cstart = nullptr, *d_cnt = nullptr,
          *d_pos = nullptr, *d_eoff = nullptr;
  uint64_t *d_seed = nullptr;
  double *d_r2 = nullptr, *d_x = nullptr, *d_y = nullptr;
  uint32_t *d_key = nullptr, *d_skey = nullptr;
  int32_t *d_src = nullptr, *d_dst = nullptr;
  xt_status s = XT_OK;
  auto h2d = [&](void *d, const void *h, size_t bytes) {
    return cuda_status(c, cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, c->stream), "H2D");
  };
  do {
    if ((s = dalloc_n(c, &d_kind, size_t(ng))) != XT_OK) break;
    if ((s = dalloc_n(c, &d_cells, size_t(ng))) != XT_OK) break;
    if ((s = dalloc_n(c, &d_n, size_t(ng))) != XT_OK) break;
    if ((s = dalloc_n(c, &d_poff, size_t(ng + 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &d_cbase, size_t(ng + 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &d_seed, size_t(ng))) != XT_OK) break;
    if ((s = dalloc_n(c, &d_r2, size_t(ng))) != XT_OK) break;
    if ((s = dalloc_n(c, &d_eoff, size_t(ng + 1))) != XT_OK) break;
    if ((s = h2d(d_kind, kind, sizeof(int32_t) * ng)) != XT_OK) break;
    if ((s = h2d(d_cells, cells.data(), sizeof(int32_t) * ng)) != XT_OK) break;
    if ((s = h2d(d_n, nvtx, sizeof(int64_t) * ng)) != XT_OK) break;
    if ((s = h2d(d_poff, poff.data(), sizeof(int64_t) * (ng + 1))) != XT_OK) break;
    if ((s = h2d(d_cbase, cbase.data(), sizeof(int64_t) * (ng + 1))) != XT_OK) break;
    if ((s = h2d(d_seed, gseed, sizeof(uint64_t) * ng)) != XT_OK) break;
    if ((s = h2d(d_r2, r2.data(), sizeof(double) * ng)) != XT_OK) break;
    // 2. points, cell keys, points sorted by cell
    if ((s = dalloc_n(c, &d_x, size_t(np))) != XT_OK) break;
    if ((s = dalloc_n(c, &d_y, size_t(np))) != XT_OK) break;
    if ((s = dalloc_n(c, &d_key, size_t(np))) != XT_OK) break;
    if ((s = dalloc_n(c, &d_skey, size_t(np))) != XT_OK) break;
    if ((s = dalloc_n(c, &d_idx, size_t(np))) != XT_OK) break;
    if ((s = dalloc_n(c, &d_order, size_t(np))) != XT_OK) break;
    k_batch_points<<<counted(c, grid_for(np, B, c->sm_count)), B, 0, c->stream>>>(
        ng, d_kind, d_poff, d_seed, d_cells, d_cbase, np, d_x, d_y, d_key, d_idx);
    {
      size_t bytes = 0;
      void *tmp = nullptr;
      cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, bytes, d_key, d_skey, d_idx, d_order, np, 0, 32,
                                                      c->stream);
      if ((s = cuda_status(c, e, "sort points")) != XT_OK) break;
      if ((s = dalloc(c, &tmp, bytes)) != XT_OK) break;
      e = cub::DeviceRadixSort::SortPairs(tmp, bytes, d_key, d_skey, d_idx, d_order, np, 0, 32, c->stream);
      dfree(c, tmp);
      if ((s = cuda_status(c, e, "sort points")) != XT_OK) break;
    }
    if ((s = dalloc_n(c, &d_cstart, size_t(ncell + 1))) != XT_OK) break;
    k_cell_starts<<<counted(c, grid_for(np + 1, B, c->sm_count)), B, 0, c->stream>>>(d_skey, np, ncell, d_cstart);
    // 3. RGG edge counts per point, their scan, per-graph edge offsets
    if ((s = dalloc_n(c, &d_cnt, size_t(np + 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &d_pos, size_t(np + 1))) != XT_OK) break;
    k_batch_rgg<false><<<counted(c, grid_for(np, B, c->sm_count)), B, 0, c->stream>>>(
        ng, d_kind, d_poff, d_r2, d_cells, d_cbase, d_x, d_y, d_order, d_cstart, np, d_cnt, nullptr, nullptr,
        nullptr);
    if ((s = cuda_status(c, cudaMemsetAsync(d_cnt + np, 0, sizeof(int64_t), c->stream), "memset")) != XT_OK) break;
    if ((s = scan_i64(c, d_cnt, d_pos, np + 1)) != XT_OK) break;
    std::vector<int64_t> pos_at(ng + 1);
    for (int64_t g = 0; g <= ng; g++)
      if ((s = cuda_status(c, cudaMemcpyAsync(&pos_at[g], d_pos + poff[g], sizeof(int64_t), cudaMemcpyDeviceToHost,
                                              c->stream), "D2H")) != XT_OK)
        break;
    if (s != XT_OK) break;
    if ((s = cuda_status(c, cudaStreamSynchronize(c->stream), "sync")) != XT_OK) break;
    h_eoff[0] = 0;
    for (int64_t g = 0; g < ng; g++) h_eoff[g + 1] = h_eoff[g] + (kind[g] == 0 ? pos_at[g + 1] - pos_at[g] : m[g]);
    const int64_t ne = h_eoff[ng];
    if ((s = h2d(d_eoff, h_eoff, sizeof(int64_t) * (ng + 1))) != XT_OK) break;
    // the RGG writer's positions: graph g's block starts at eoff[g]
    {
      std::vector<int64_t> shift(ng);
      for (int64_t g = 0; g < ng; g++) shift[g] = h_eoff[g] - pos_at[g];
      int64_t *d_shift = nullptr;
      if ((s = dalloc_n(c, &d_shift, size_t(ng))) != XT_OK) break;
      s = h2d(d_shift, shift.data(), sizeof(int64_t) * ng);
      if (s == XT_OK) {
        k_shift_pos<<<counted(c, grid_for(np, B, c->sm_count)), B, 0, c->stream>>>(ng, d_poff, d_shift, np, d_pos);
        s = cuda_status(c, cudaGetLastError(), "shift");
      }
      dfree(c, d_shift);
      if (s != XT_OK) break;
    }
    // 4. edges
    if ((s = dalloc_n(c, &d_src, size_t(ne > 0 ? ne : 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &d_dst, size_t(ne > 0 ? ne : 1))) != XT_OK) break;
    if (ne > 0) {
      k_batch_er<<<counted(c, grid_for(ne, B, c->sm_count)), B, 0, c->stream>>>(ng, d_kind, d_n, d_seed, d_eoff, ne,
                                                                                d_src, d_dst);
      k_batch_rgg<true><<<counted(c, grid_for(np, B, c->sm_count)), B, 0, c->stream>>>(
          ng, d_kind, d_poff, d_r2, d_cells, d_cbase, d_x, d_y, d_order, d_cstart, np, nullptr, d_pos, d_src, d_dst);
    }
    if ((s = cuda_status(c, cudaGetLastError(), "batch edges")) != XT_OK) break;
    if ((s = cuda_status(c, cudaStreamSynchronize(c->stream), "sync")) != XT_OK) break;
    *d_src_out = d_src;
    *d_dst_out = d_dst;
    d_src = d_dst = nullptr;
  } while (0);
  for (void *p : {(void *)d_kind, (void *)d_cells, (void *)d_order, (void *)d_idx, (void *)d_n, (void *)d_poff,
                  (void *)d_cbase, (void *)d_cstart, (void *)d_cnt, (void *)d_pos, (void *)d_eoff, (void *)d_seed,
                  (void *)d_r2, (void *)d_x, (void *)d_y, (void *)d_key, (void *)d_skey, (void *)d_src,
                  (void *)d_dst})
    dfree(c, p);
  return s;
}

}  // namespace xt

// ---- capture, tuning, autotuner ----------------------------------------------

namespace xt {

xt_status capture_count(Graph *g) {
  Ctx *c = g->ctx;
  if (!g->plan) XT_TRY(make_plan(g));
  if (g->exec) {
    cudaGraphExecDestroy(g->exec);
    g->exec = nullptr;
  }
  if (!g->d_res) XT_TRY(dalloc_n(c, &g->d_res, size_t(1 + g->n_groups)));
  XT_CUDA(c, cudaStreamSynchronize(c->stream));  // the allocation is complete before capture
  // record on a private stream (the context's may be the legacy default
  // stream, which cannot capture); the graph is replayed on the context's
  cudaStream_t cap = nullptr;
  XT_CUDA(c, cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
  cudaStream_t saved = c->stream;
  c->stream = cap;
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
  xt_status s = XT_OK;
  const int64_t l0 = c->launches;
  if (e == cudaSuccess) {
    s = count_graph(g, g->d_res, nullptr, g->n_groups > 0 ? g->d_res + 1 : nullptr);
    e = cudaStreamEndCapture(cap, &graph);
  }
  // recorded kernels run (and are counted) at each replay, not here
  g->exec_kernels = c->launches - l0;
  c->launches = l0;
  c->stream = saved;
  cudaStreamDestroy(cap);
  if (s != XT_OK) {
    if (graph) cudaGraphDestroy(graph);
    return s;
  }
  XT_CUDA(c, e);
  e = cudaGraphInstantiate(&g->exec, graph, 0);
  cudaGraphDestroy(graph);
  XT_CUDA(c, e);
  return XT_OK;
}

// runs the count into g->d_res (replaying the captured graph when there is one)
xt_status run_count_res(Graph *g) {
  Ctx *c = g->ctx;
  if (g->exec) {
    XT_CUDA(c, cudaGraphLaunch(g->exec, c->stream));
    c->launches += g->exec_kernels;
    return XT_OK;
  }
  if (!g->d_res) XT_TRY(dalloc_n(c, &g->d_res, size_t(1 + g->n_groups)));
  return count_graph(g, g->d_res, nullptr, g->n_groups > 0 ? g->d_res + 1 : nullptr);
}

xt_status set_tiers(Graph *g, int64_t lane_work, int64_t warp_work) {
  const bool was_captured = g->exec != nullptr;
  g->tier_lane_work = lane_work >= 0 ? lane_work : -1;
  g->tier_warp_work = warp_work >= 0 ? warp_work : -1;
  XT_TRY(make_plan(g));
  if (was_captured) XT_TRY(capture_count(g));
  return XT_OK;
}

xt_status set_prefetch(Graph *g, int on) {
  g->prefetch_suffix = on ? 1 : 0;
  if (g->exec) XT_TRY(capture_count(g));  // the launch inside the captured graph changes
  return XT_OK;
}

static xt_status set_lane_merge(Graph *g, int on) {
  g->lane_merge = on ? 1 : 0;
  if (g->exec) XT_TRY(capture_count(g));  // the launch's arguments inside the captured graph change
  return XT_OK;
}

static xt_status set_claim(Graph *g, int claim) {
  g->claim_block = claim;
  if (g->exec) XT_TRY(capture_count(g));  // the launch's arguments inside the captured graph change
  return XT_OK;
}

static xt_status set_cluster(Graph *g, int on) {
  const bool was_captured = g->exec != nullptr;
  g->cluster_tier = on ? 1 : 0;
  XT_TRY(make_plan(g));
  if (was_captured) XT_TRY(capture_count(g));
  return XT_OK;
}

xt_status set_tuning(Graph *g, int64_t block_work, int64_t warp_work, int64_t bitmap_bits) {
  const bool was_captured = g->exec != nullptr;
  g->tune_block_work = block_work > 0 ? block_work : 0;
  g->tune_warp_work = warp_work > 0 ? warp_work : 0;
  g->tune_bitmap_bits = bitmap_bits > 0 ? bitmap_bits : 0;
  XT_TRY(make_plan(g));
  if (was_captured) XT_TRY(capture_count(g));
  return XT_OK;
}

static xt_status time_count(Graph *g, int reps, double *ms) {
  Ctx *c = g->ctx;
  cudaEvent_t a = nullptr, b = nullptr;
  XT_CUDA(c, cudaEventCreate(&a));
  cudaError_t e = cudaEventCreate(&b);
  if (e != cudaSuccess) {
    cudaEventDestroy(a);
    return cuda_status(c, e, "event");
  }
  xt_status s = run_count_res(g);  // warm-up
  float best = 1e30f;
  for (int r = 0; r < reps && s == XT_OK; r++) {
    cudaEventRecord(a, c->stream);
    s = run_count_res(g);
    cudaEventRecord(b, c->stream);
    if (s == XT_OK) s = cuda_status(c, cudaEventSynchronize(b), "event");
    float t = 0;
    if (s == XT_OK) cudaEventElapsedTime(&t, a, b);
    best = std::min(best, t);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *ms = best;
  return s;
}

static std::string tune_key(const Graph *g) {
  cudaDeviceProp p;
  cudaGetDeviceProperties(&p, g->ctx->device);
  auto lg = [](int64_t x) {
    int b = 0;
    while (x > 1) {
      x >>= 1;
      b++;
    }
    return b;
  };
  char buf[512];
  // the schedule revision keeps timings of an older kernel from being reused
  snprintf(buf, sizeof buf, "sched10|%s|sm%d|orient%d|nv2^%d|ne2^%d|work2^%d|groups%lld", p.name, p.multiProcessorCount,
           g->orient, lg(g->nv), lg(g->ne), lg(g->stream_work), (long long)g->n_groups);
  for (char *q = buf; *q; q++)
    if (*q == ' ') *q = '_';
  return buf;
}

// Coordinate search over the schedule: the CTA task size, the warp-task work
// limit and the largest member id range kept as a bitmap (beyond it the hash
// is used), each swept with the others held, the best kept; then the bulk
// suffix prefetch on and off, the lane tier's merge, and the warp tasks
// claimed per atomic (1, 4, 16). Results are cached per (GPU, graph class)
// in a text file when a path is given, so a second run of the same class of
// graph skips the search.
xt_status autotune(Graph *g, int reps, const char *cache_path, std::string *report) {
  const std::string key = tune_key(g);
  if (cache_path && *cache_path) {
    if (FILE *f = fopen(cache_path, "r")) {
      char line[512];
      while (fgets(line, sizeof line, f)) {
        char k[300];
        long long bw, ww, bb;
        int pf, lm, cl;
        double ms;
        if (sscanf(line, "%299s %lld %lld %lld %d %d %d %lf", k, &bw, &ww, &bb, &pf, &lm, &cl, &ms) == 8 &&
            key == k) {
          fclose(f);
          if (report) *report = "{\"cached\": true, \"key\": \"" + key + "\"}";
          XT_TRY(set_prefetch(g, pf));
          XT_TRY(set_lane_merge(g, lm));
          XT_TRY(set_claim(g, cl));
          return set_tuning(g, bw, ww, bb);
        }
      }
      fclose(f);
    }
  }
  int64_t best[3] = {0, 0, 0};
  double best_ms = 0;
  XT_TRY(set_prefetch(g, 0));
  XT_TRY(set_lane_merge(g, 0));
  XT_TRY(set_claim(g, 0));
  XT_TRY(set_tuning(g, 0, 0, 0));
  XT_TRY(time_count(g, reps, &best_ms));
  std::string rep = "{\"key\": \"" + key + "\", \"trials\": [";
  char buf[160];
  snprintf(buf, sizeof buf, "{\"block_work\": 0, \"warp_work\": 0, \"bitmap_bits\": 0, \"ms\": %.4f}", best_ms);
  rep += buf;
  const std::vector<int64_t> options[3] = {
      {int64_t(1) << 14, int64_t(1) << 16, int64_t(1) << 17, int64_t(1) << 18, int64_t(1) << 20},
      {1024, 4096, 8192, 16384},
      {int64_t(1) << 13, int64_t(1) << 16, int64_t(1) << 18}};
  for (int dim = 0; dim < 3; dim++) {
    for (int64_t opt : options[dim]) {
      int64_t p[3] = {best[0], best[1], best[2]};
      p[dim] = opt;
      XT_TRY(set_tuning(g, p[0], p[1], p[2]));
      double ms = 0;
      XT_TRY(time_count(g, reps, &ms));
      snprintf(buf, sizeof buf, ", {\"block_work\": %lld, \"warp_work\": %lld, \"bitmap_bits\": %lld, \"ms\": %.4f}",
               (long long)p[0], (long long)p[1], (long long)p[2], ms);
      rep += buf;
      if (ms < best_ms) {
        best_ms = ms;
        best[dim] = opt;
      }
    }
  }
  XT_TRY(set_tuning(g, best[0], best[1], best[2]));
  int best_pf = 0;
  {
    XT_TRY(set_prefetch(g, 1));
    double ms = 0;
    XT_TRY(time_count(g, reps, &ms));
    snprintf(buf, sizeof buf, ", {\"block_work\": %lld, \"warp_work\": %lld, \"bitmap_bits\": %lld, \"prefetch\": 1, "
             "\"ms\": %.4f}", (long long)best[0], (long long)best[1], (long long)best[2], ms);
    rep += buf;
    if (ms < best_ms) {
      best_ms = ms;
      best_pf = 1;
    }
    XT_TRY(set_prefetch(g, best_pf));
  }
  // the lane tier's intersection: binary search or two-pointer merge (only
  // where the plan has lane tasks)
  int best_lm = 0;
  if (lane_task_count(g) > 0) {
    XT_TRY(set_lane_merge(g, 1));
    double ms = 0;
    XT_TRY(time_count(g, reps, &ms));
    snprintf(buf, sizeof buf, ", {\"lane_merge\": 1, \"ms\": %.4f}", ms);
    rep += buf;
    if (ms < best_ms) {
      best_ms = ms;
      best_lm = 1;
    }
    XT_TRY(set_lane_merge(g, best_lm));
  }
  // warp (and lane) tasks claimed per atomic on their cursor: 0 is the
  // automatic choice timed above
  int best_cl = 0;
  for (int cl : {1, 4, 16}) {
    XT_TRY(set_claim(g, cl));
    double ms = 0;
    XT_TRY(time_count(g, reps, &ms));
    snprintf(buf, sizeof buf, ", {\"claim\": %d, \"ms\": %.4f}", cl, ms);
    rep += buf;
    if (ms < best_ms) {
      best_ms = ms;
      best_cl = cl;
    }
  }
  XT_TRY(set_claim(g, best_cl));
  snprintf(buf, sizeof buf,
           "], \"best\": {\"block_work\": %lld, \"warp_work\": %lld, \"bitmap_bits\": %lld, \"prefetch\": %d, "
           "\"lane_merge\": %d, \"claim\": %d, \"ms\": %.4f}}",
           (long long)best[0], (long long)best[1], (long long)best[2], best_pf, best_lm, best_cl, best_ms);
  rep += buf;
  if (report) *report = rep;
  if (cache_path && *cache_path) {
    if (FILE *f = fopen(cache_path, "a")) {
      fprintf(f, "%s %lld %lld %lld %d %d %d %.4f\n", key.c_str(), (long long)best[0], (long long)best[1],
              (long long)best[2], best_pf, best_lm, best_cl, best_ms);
      fclose(f);
    }
  }
  return XT_OK;
}

}  // namespace xt

// ---- C ABI --------------------------------------------------------------------

using namespace xt;

extern "C" {

xt_status xt_batch_spec(int64_t n_graphs, uint64_t seed, int32_t *kind, int64_t *n, double *mean_deg,
                        uint64_t *graph_seed) {
  if (n_graphs < 1 || !kind || !n || !mean_deg || !graph_seed) return XT_ERR_INVALID;
  for (int64_t i = 0; i < n_graphs; i++) {
    const uint64_t r0 = crand(seed, kStreamBatch, 4u * uint64_t(i)), r1 = crand(seed, kStreamBatch, 4u * uint64_t(i) + 1u);
    const uint64_t r2 = crand(seed, kStreamBatch, 4u * uint64_t(i) + 2u), r3 = crand(seed, kStreamBatch, 4u * uint64_t(i) + 3u);
    kind[i] = int32_t(i & 1);  // half random geometric, half Erdos-Renyi
    // vertex count log-uniform in [256, 65536): a uniform octave, uniform inside it
    const uint64_t oct = r0 >> 61, base = uint64_t(256) << oct;
    n[i] = int64_t(base + uint64_t((unsigned __int128)r1 * base >> 64));
    // mean degree log-uniform in [8, 64) the same way
    const uint64_t doct = uint64_t((unsigned __int128)r2 * 3u >> 64);
    mean_deg[i] = double(uint64_t(8) << doct) * (1.0 + double(r3 >> 11) * (1.0 / 9007199254740992.0));
    graph_seed[i] = mix64(seed ^ (0x9e3779b97f4a7c15ULL * uint64_t(i + 1)));
  }
  return XT_OK;
}

xt_status xt_gen_batch(xt_ctx *ctx, int64_t n_graphs, const int32_t *kind, const int64_t *n, const double *mean_deg,
                       const uint64_t *graph_seed, int64_t *edge_offsets, int32_t **d_src, int32_t **d_dst) {
  if (!ctx || n_graphs < 1 || !kind || !n || !mean_deg || !graph_seed || !edge_offsets || !d_src || !d_dst)
    return XT_ERR_INVALID;
  cudaSetDevice(ctx->c.device);
  *d_src = *d_dst = nullptr;
  return gen_batch(&ctx->c, n_graphs, kind, n, mean_deg, graph_seed, edge_offsets, d_src, d_dst);
}

xt_status xt_device_free(xt_ctx *ctx, void *p) {
  if (!ctx) return XT_ERR_INVALID;
  cudaSetDevice(ctx->c.device);
  dfree(&ctx->c, p);
  XT_CUDA(&ctx->c, cudaStreamSynchronize(ctx->c.stream));
  return XT_OK;
}

xt_status xt_graph_from_device_batch(xt_ctx *ctx, int64_t n_graphs, const int64_t *vertex_offsets,
                                     const int64_t *edge_offsets, const int32_t *d_src, const int32_t *d_dst,
                                     int orient, xt_graph **out) {
  if (!ctx || !out || !vertex_offsets || !edge_offsets) return XT_ERR_INVALID;
  *out = nullptr;
  Ctx *c = &ctx->c;
  cudaSetDevice(c->device);
  xt_graph *gr = new (std::nothrow) xt_graph();
  if (!gr) return XT_ERR_OOM;
  xt_status s = build_batch(c, n_graphs, vertex_offsets, edge_offsets, d_src, d_dst, orient, &gr->g);
  if (s == XT_OK) s = make_plan(&gr->g);
  if (s == XT_OK) s = cuda_status(c, cudaStreamSynchronize(c->stream), "build");
  if (s != XT_OK) {
    free_graph_device(&gr->g);
    cudaStreamSynchronize(c->stream);
    delete gr;
    return s;
  }
  *out = gr;
  return XT_OK;
}

xt_status xt_graph_from_batch(xt_ctx *ctx, int64_t n_graphs, const int64_t *vertex_offsets,
                              const int64_t *edge_offsets, const int32_t *src, const int32_t *dst, int orient,
                              xt_graph **out) {
  if (!ctx || !out || !vertex_offsets || !edge_offsets || n_graphs < 1) return XT_ERR_INVALID;
  Ctx *c = &ctx->c;
  cudaSetDevice(c->device);
  const int64_t ne = edge_offsets[n_graphs];
  if (ne < 0 || (ne > 0 && (!src || !dst))) return XT_ERR_INVALID;
  int32_t *ds = nullptr, *dd = nullptr;
  XT_TRY(dalloc_n(c, &ds, size_t(ne > 0 ? ne : 1)));
  xt_status s = dalloc_n(c, &dd, size_t(ne > 0 ? ne : 1));
  if (s == XT_OK && ne > 0) {
    s = cuda_status(c, cudaMemcpyAsync(ds, src, sizeof(int32_t) * ne, cudaMemcpyHostToDevice, c->stream), "H2D");
    if (s == XT_OK)
      s = cuda_status(c, cudaMemcpyAsync(dd, dst, sizeof(int32_t) * ne, cudaMemcpyHostToDevice, c->stream), "H2D");
  }
  if (s == XT_OK) s = xt_graph_from_device_batch(ctx, n_graphs, vertex_offsets, edge_offsets, ds, dd, orient, out);
  dfree(c, ds);
  dfree(c, dd);
  return s;
}

xt_status xt_count_groups_async(xt_graph *gr, int64_t *d_total, int64_t *d_per_group) {
  if (!gr || !d_total) return XT_ERR_INVALID;
  Graph &g = gr->g;
  cudaSetDevice(g.ctx->device);
  XT_TRY(run_count_res(&g));
  Ctx *c = g.ctx;
  XT_CUDA(c, cudaMemcpyAsync(d_total, g.d_res, sizeof(int64_t), cudaMemcpyDeviceToDevice, c->stream));
  if (d_per_group && g.n_groups > 0)
    XT_CUDA(c, cudaMemcpyAsync(d_per_group, g.d_res + 1, sizeof(int64_t) * g.n_groups, cudaMemcpyDeviceToDevice,
                               c->stream));
  return XT_OK;
}

xt_status xt_count_groups(xt_graph *gr, int64_t *total, int64_t *per_group) {
  if (!gr || !total) return XT_ERR_INVALID;
  Graph &g = gr->g;
  Ctx *c = g.ctx;
  cudaSetDevice(c->device);
  XT_TRY(run_count_res(&g));
  XT_CUDA(c, cudaMemcpyAsync(total, g.d_res, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
  if (per_group && g.n_groups > 0)
    XT_CUDA(c, cudaMemcpyAsync(per_group, g.d_res + 1, sizeof(int64_t) * g.n_groups, cudaMemcpyDeviceToHost,
                               c->stream));
  XT_CUDA(c, cudaStreamSynchronize(c->stream));
  return count_status(c);
}

int64_t xt_graph_groups(const xt_graph *gr) { return gr ? gr->g.n_groups : -1; }

xt_status xt_batch_count(xt_ctx *ctx, int64_t n_graphs, const int64_t *vertex_offsets, const int64_t *edge_offsets,
                         const int32_t *src, const int32_t *dst, int orient, int64_t *total, int64_t *per_graph) {
  if (!ctx || !total) return XT_ERR_INVALID;
  xt_graph *g = nullptr;
  XT_TRY(xt_graph_from_batch(ctx, n_graphs, vertex_offsets, edge_offsets, src, dst, orient, &g));
  const xt_status s = xt_count_groups(g, total, per_graph);
  xt_graph_free(g);
  return s;
}

xt_status xt_graph_capture(xt_graph *gr) {
  if (!gr) return XT_ERR_INVALID;
  cudaSetDevice(gr->g.ctx->device);
  return capture_count(&gr->g);
}

xt_status xt_graph_set_tuning(xt_graph *gr, int64_t block_work, int64_t warp_work, int64_t bitmap_bits) {
  if (!gr) return XT_ERR_INVALID;
  cudaSetDevice(gr->g.ctx->device);
  return set_tuning(&gr->g, block_work, warp_work, bitmap_bits);
}

xt_status xt_graph_set_tiers(xt_graph *gr, int64_t lane_work, int64_t warp_work) {
  if (!gr) return XT_ERR_INVALID;
  cudaSetDevice(gr->g.ctx->device);
  return set_tiers(&gr->g, lane_work, warp_work);
}

xt_status xt_graph_debug_cuckoo_iters(xt_graph *gr, int iters) {
  if (!gr || !gr->g.ctx) return XT_ERR_INVALID;
  gr->g.cuckoo_iters = iters < 0 ? -1 : iters;
  if (gr->g.exec) {
    cudaSetDevice(gr->g.ctx->device);
    return capture_count(&gr->g);
  }
  return XT_OK;
}

xt_status xt_graph_set_prefetch(xt_graph *gr, int on) {
  if (!gr || !gr->g.ctx) return XT_ERR_INVALID;
  cudaSetDevice(gr->g.ctx->device);
  return set_prefetch(&gr->g, on);
}

xt_status xt_graph_set_lane_intersect(xt_graph *gr, int kind) {
  if (!gr || !gr->g.ctx || (kind != XT_LANE_BSEARCH && kind != XT_LANE_MERGE)) return XT_ERR_INVALID;
  cudaSetDevice(gr->g.ctx->device);
  return set_lane_merge(&gr->g, kind == XT_LANE_MERGE);
}

xt_status xt_graph_set_claim(xt_graph *gr, int claim) {
  if (!gr || !gr->g.ctx || claim < 0 || claim > 64) return XT_ERR_INVALID;
  cudaSetDevice(gr->g.ctx->device);
  return set_claim(&gr->g, claim);
}

xt_status xt_graph_set_cluster(xt_graph *gr, int on) {
  if (!gr || !gr->g.ctx) return XT_ERR_INVALID;
  cudaSetDevice(gr->g.ctx->device);
  return set_cluster(&gr->g, on);
}

xt_status xt_graph_autotune(xt_graph *gr, int reps, const char *cache_path, char *report, int64_t report_len) {
  if (!gr || reps < 1) return XT_ERR_INVALID;
  cudaSetDevice(gr->g.ctx->device);
  std::string rep;
  xt_status s = autotune(&gr->g, reps, cache_path, &rep);
  if (report && report_len > 0) {
    const size_t k = std::min(rep.size(), size_t(report_len - 1));
    std::memcpy(report, rep.data(), k);
    report[k] = 0;
  }
  return s;
}

}  // extern "C"
