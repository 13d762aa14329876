// GPU CSR builder: canonicalise (drop self loops, symmetrise, dedup), orient
// each undirected edge from the lower to the higher rank, and emit the
// oriented out-CSR (int64 offsets, int32 ascending columns) together with
// its transpose (the in-lists N-(v)) that the head-grouped count streams.
//
// Reference behaviour replaced: the reference trusts its input CSR
// (graph.hpp:294-395 reads it verbatim; a duplicated pair over-counts) and
// orients implicitly by vertex id inside the count loop (xxtric.hpp:165,
// counting.cu:619). Here the builder makes any edge list canonical first, so
// the count of a canonical input equals the reference's count on it.
#include <cub/cub.cuh>

#include "xt_internal.cuh"

namespace xt {

static int bits_for(int64_t nv) {
  int b = 1;
  while ((int64_t(1) << b) < nv) b++;
  return b;
}

static unsigned grid_for(int64_t n, int block, int sm_count) {
  int64_t g = (n + block - 1) / block;
  int64_t cap = int64_t(sm_count) * 32;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (unsigned)g;
}

// key = (min << b) | max; self loops keep min == max and are dropped later.
__global__ void k_edge_keys(const int32_t *__restrict__ src, const int32_t *__restrict__ dst, int64_t ne,
                            int64_t nv, int b, uint64_t *__restrict__ keys, int *__restrict__ err) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < ne; i += int64_t(gridDim.x) * blockDim.x) {
    int64_t s = src[i], d = dst[i];
    if (s < 0 || d < 0 || s >= nv || d >= nv) {
      atomicOr(err, 1);
      s = 0;
      d = 0;
    }
    uint64_t lo = uint64_t(s < d ? s : d), hi = uint64_t(s < d ? d : s);
    keys[i] = (lo << b) | hi;
  }
}

__global__ void k_unique_flags(const uint64_t *__restrict__ keys, int64_t n, int b, uint8_t *__restrict__ flags) {
  const uint64_t mask = (uint64_t(1) << b) - 1;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    uint64_t k = keys[i];
    bool first = (i == 0) || (keys[i - 1] != k);
    flags[i] = (first && ((k >> b) != (k & mask))) ? 1 : 0;
  }
}

__global__ void k_degrees(const uint64_t *__restrict__ uniq, int64_t m, int b, int32_t *__restrict__ deg) {
  const uint64_t mask = (uint64_t(1) << b) - 1;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < m; i += int64_t(gridDim.x) * blockDim.x) {
    uint64_t k = uniq[i];
    atomicAdd(&deg[k >> b], 1);
    atomicAdd(&deg[k & mask], 1);
  }
}

__device__ __forceinline__ bool rank_less(int64_t a, int64_t b_, const int32_t *__restrict__ deg) {
  int32_t da = deg[a], db = deg[b_];
  return da < db || (da == db && a < b_);
}

// (lo,hi) -> (src,dst) by (degree, id) rank
__global__ void k_orient_degree(uint64_t *__restrict__ keys, int64_t m, int b, const int32_t *__restrict__ deg) {
  const uint64_t mask = (uint64_t(1) << b) - 1;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < m; i += int64_t(gridDim.x) * blockDim.x) {
    uint64_t k = keys[i];
    int64_t lo = int64_t(k >> b), hi = int64_t(k & mask);
    if (!rank_less(lo, hi, deg)) keys[i] = (uint64_t(hi) << b) | uint64_t(lo);
  }
}

// (src,dst) -> (dst,src)
__global__ void k_swap_keys(const uint64_t *__restrict__ in, int64_t m, int b, uint64_t *__restrict__ out) {
  const uint64_t mask = (uint64_t(1) << b) - 1;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < m; i += int64_t(gridDim.x) * blockDim.x) {
    uint64_t k = in[i];
    out[i] = ((k & mask) << b) | (k >> b);
  }
}

// Sorted keys (row << b | col) -> CSR. off[u] = index of the first key whose
// row is >= u: thread i writes the rows in (row[i-1], row[i]] so every entry
// of off is written exactly once, deterministically.
__global__ void k_finish_csr(const uint64_t *__restrict__ keys, int64_t m, int64_t nv, int b,
                             int64_t *__restrict__ off, int32_t *__restrict__ col) {
  const uint64_t mask = (uint64_t(1) << b) - 1;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i <= m; i += int64_t(gridDim.x) * blockDim.x) {
    int64_t prev = (i == 0) ? -1 : int64_t(keys[i - 1] >> b);
    int64_t cur = (i == m) ? nv : int64_t(keys[i] >> b);
    for (int64_t u = prev + 1; u <= cur; u++) off[u] = i;
    if (i < m) col[i] = int32_t(keys[i] & mask);
  }
}

// CSR input: row index of every entry (warp per row) and range checks.
__global__ void k_csr_rows(const int64_t *__restrict__ off, int64_t nv, int64_t ne_in, int32_t *__restrict__ rows,
                           int *__restrict__ err) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t u = warp; u < nv; u += nwarps) {
    int64_t e0 = off[u], e1 = off[u + 1];
    if (e0 < 0 || e1 < e0 || e1 > ne_in) {
      if (lane == 0) atomicOr(err, 2);
      continue;
    }
    for (int64_t e = e0 + lane; e < e1; e += 32) rows[e] = int32_t(u);
  }
}

__global__ void k_csr_tails32(const int64_t *__restrict__ tails, int64_t n, int64_t nv, int32_t *__restrict__ out,
                              int *__restrict__ err) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    int64_t t = tails[i];
    if (t < 0 || t >= nv) {
      atomicOr(err, 1);
      t = 0;
    }
    out[i] = int32_t(t);
  }
}

// Canonical CSR input: keep entry (u,t) when u ranks below t; the kept
// entries stay in (row, column) order, so no sort is needed.
__global__ void k_csr_orient_keys(const int32_t *__restrict__ rows, const int32_t *__restrict__ tails, int64_t n,
                                  const int64_t *__restrict__ off, int orient, int b, uint64_t *__restrict__ keys,
                                  uint8_t *__restrict__ flags) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    int64_t u = rows[i], t = tails[i];
    bool keep;
    if (orient == XT_ORIENT_ID) {
      keep = u < t;
    } else {
      int64_t du = off[u + 1] - off[u], dt = off[t + 1] - off[t];
      keep = du < dt || (du == dt && u < t);
    }
    flags[i] = keep ? 1 : 0;
    keys[i] = (uint64_t(u) << b) | uint64_t(t);
  }
}

__global__ void k_degree_from_off(const int64_t *__restrict__ off, int64_t nv, int32_t *__restrict__ deg) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nv; i += int64_t(gridDim.x) * blockDim.x)
    deg[i] = int32_t(off[i + 1] - off[i]);
}

// ---------------------------------------------------------------------------

static xt_status sort_keys(Ctx *c, const uint64_t *in, uint64_t *out, int64_t n, int end_bit) {
  size_t bytes = 0;
  XT_CUDA(c, cub::DeviceRadixSort::SortKeys(nullptr, bytes, in, out, n, 0, end_bit, c->stream));
  void *tmp = nullptr;
  XT_TRY(dalloc(c, &tmp, bytes));
  cudaError_t e = cub::DeviceRadixSort::SortKeys(tmp, bytes, in, out, n, 0, end_bit, c->stream);
  dfree(c, tmp);
  XT_CUDA(c, e);
  return XT_OK;
}

static xt_status select_flagged(Ctx *c, const uint64_t *in, const uint8_t *flags, uint64_t *out, int64_t n,
                                int64_t *m_out) {
  int64_t *d_num = nullptr;
  XT_TRY(dalloc_n(c, &d_num, 1));
  size_t bytes = 0;
  cudaError_t e = cub::DeviceSelect::Flagged(nullptr, bytes, in, flags, out, d_num, n, c->stream);
  if (e != cudaSuccess) {
    dfree(c, d_num);
    return cuda_status(c, e, "DeviceSelect::Flagged");
  }
  void *tmp = nullptr;
  xt_status s = dalloc(c, &tmp, bytes);
  if (s != XT_OK) {
    dfree(c, d_num);
    return s;
  }
  e = cub::DeviceSelect::Flagged(tmp, bytes, in, flags, out, d_num, n, c->stream);
  dfree(c, tmp);
  if (e == cudaSuccess) e = cudaMemcpyAsync(m_out, d_num, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  dfree(c, d_num);
  XT_CUDA(c, e);
  return XT_OK;
}

static xt_status check_err(Ctx *c, const char *what) {
  int h = 0;
  XT_CUDA(c, cudaMemcpyAsync(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  XT_CUDA(c, cudaStreamSynchronize(c->stream));
  if (h) {
    XT_CUDA(c, cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
    return set_error(c, XT_ERR_INVALID,
                     std::string(what) + ((h & 1) ? ": vertex id outside [0,nv)" : ": offsets not monotone in [0,ne]"));
  }
  return XT_OK;
}

// Sorted oriented keys (src<<b|dst, m of them) -> out-CSR and in-CSR.
static xt_status finish_graph(Ctx *c, uint64_t *okeys, int64_t m, int64_t nv, int b, Graph *g) {
  const int B = 256;
  g->ne = m;
  XT_TRY(dalloc_n(c, &g->d_off, size_t(nv + 1)));
  XT_TRY(dalloc_n(c, &g->d_col, size_t(m > 0 ? m : 1)));
  k_finish_csr<<<counted(c, grid_for(m + 1, B, c->sm_count)), B, 0, c->stream>>>(okeys, m, nv, b, g->d_off, g->d_col);
  XT_CUDA(c, cudaGetLastError());
  // transpose: sort (dst<<b|src)
  uint64_t *t0 = nullptr, *t1 = nullptr;
  XT_TRY(dalloc_n(c, &t0, size_t(m > 0 ? m : 1)));
  xt_status s = dalloc_n(c, &t1, size_t(m > 0 ? m : 1));
  if (s != XT_OK) {
    dfree(c, t0);
    return s;
  }
  k_swap_keys<<<counted(c, grid_for(m, B, c->sm_count)), B, 0, c->stream>>>(okeys, m, b, t0);
  s = (m > 0) ? sort_keys(c, t0, t1, m, 2 * b) : XT_OK;
  dfree(c, t0);
  if (s != XT_OK) {
    dfree(c, t1);
    return s;
  }
  s = dalloc_n(c, &g->d_ioff, size_t(nv + 1));
  if (s == XT_OK) s = dalloc_n(c, &g->d_icol, size_t(m > 0 ? m : 1));
  if (s == XT_OK) {
    k_finish_csr<<<counted(c, grid_for(m + 1, B, c->sm_count)), B, 0, c->stream>>>(t1, m, nv, b, g->d_ioff, g->d_icol);
    s = cuda_status(c, cudaGetLastError(), "k_finish_csr");
  }
  dfree(c, t1);
  return s;
}

xt_status build_from_edges(Ctx *c, int64_t nv, int64_t ne, const int32_t *d_src, const int32_t *d_dst, int orient,
                           Graph *g) {
  if (nv < 1 || ne < 0) return set_error(c, XT_ERR_INVALID, "nv must be >= 1 and ne >= 0");
  if (nv > (int64_t(1) << 31) - 1) return set_error(c, XT_ERR_OVERFLOW, "nv must be below 2^31");
  if (orient != XT_ORIENT_ID && orient != XT_ORIENT_DEGREE) return set_error(c, XT_ERR_INVALID, "bad orientation");
  g->ctx = c;
  g->nv = nv;
  g->n_input = ne;
  g->orient = orient;
  const int b = bits_for(nv);
  const int B = 256;
  uint64_t *k0 = nullptr, *k1 = nullptr;
  uint8_t *flags = nullptr;
  int32_t *deg = nullptr;
  int64_t m = 0;
  xt_status s = XT_OK;
  const size_t n1 = size_t(ne > 0 ? ne : 1);
  do {
    if ((s = dalloc_n(c, &k0, n1)) != XT_OK) break;
    if ((s = dalloc_n(c, &k1, n1)) != XT_OK) break;
    if ((s = dalloc_n(c, &flags, n1)) != XT_OK) break;
    if (ne > 0) {
      k_edge_keys<<<counted(c, grid_for(ne, B, c->sm_count)), B, 0, c->stream>>>(d_src, d_dst, ne, nv, b, k0, c->d_err);
      if ((s = cuda_status(c, cudaGetLastError(), "k_edge_keys")) != XT_OK) break;
      if ((s = check_err(c, "edge list")) != XT_OK) break;
      if ((s = sort_keys(c, k0, k1, ne, 2 * b)) != XT_OK) break;
      k_unique_flags<<<counted(c, grid_for(ne, B, c->sm_count)), B, 0, c->stream>>>(k1, ne, b, flags);
      if ((s = select_flagged(c, k1, flags, k0, ne, &m)) != XT_OK) break;
    }
    // k0[0..m) = unique undirected (lo,hi), sorted
    if ((s = dalloc_n(c, &deg, size_t(nv))) != XT_OK) break;
    if ((s = cuda_status(c, cudaMemsetAsync(deg, 0, sizeof(int32_t) * nv, c->stream), "memset")) != XT_OK) break;
    k_degrees<<<counted(c, grid_for(m, B, c->sm_count)), B, 0, c->stream>>>(k0, m, b, deg);
    if (orient == XT_ORIENT_DEGREE && m > 0) {
      k_orient_degree<<<counted(c, grid_for(m, B, c->sm_count)), B, 0, c->stream>>>(k0, m, b, deg);
      if ((s = sort_keys(c, k0, k1, m, 2 * b)) != XT_OK) break;
      std::swap(k0, k1);
    }
    if ((s = cuda_status(c, cudaGetLastError(), "orient")) != XT_OK) break;
    g->d_deg = deg;
    deg = nullptr;
    s = finish_graph(c, k0, m, nv, b, g);
  } while (0);
  dfree(c, k0);
  dfree(c, k1);
  dfree(c, flags);
  dfree(c, deg);
  if (s != XT_OK) free_graph_device(g);
  return s;
}

xt_status build_from_csr(Ctx *c, int64_t nv, const int64_t *d_off, const int64_t *d_tails, bool canonical,
                         int orient, Graph *g) {
  if (nv < 1) return set_error(c, XT_ERR_INVALID, "nv must be >= 1");
  if (nv > (int64_t(1) << 31) - 1) return set_error(c, XT_ERR_OVERFLOW, "nv must be below 2^31");
  int64_t ne_in = 0;
  XT_CUDA(c, cudaMemcpyAsync(&ne_in, d_off + nv, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
  XT_CUDA(c, cudaStreamSynchronize(c->stream));
  if (ne_in < 0) return set_error(c, XT_ERR_INVALID, "offsets[nv] is negative");
  const int B = 256;
  int32_t *rows = nullptr, *t32 = nullptr;
  xt_status s = XT_OK;
  const size_t n1 = size_t(ne_in > 0 ? ne_in : 1);
  do {
    if ((s = dalloc_n(c, &rows, n1)) != XT_OK) break;
    if ((s = dalloc_n(c, &t32, n1)) != XT_OK) break;
    k_csr_rows<<<counted(c, grid_for(nv * 32, B, c->sm_count)), B, 0, c->stream>>>(d_off, nv, ne_in, rows, c->d_err);
    k_csr_tails32<<<counted(c, grid_for(ne_in, B, c->sm_count)), B, 0, c->stream>>>(d_tails, ne_in, nv, t32, c->d_err);
    if ((s = cuda_status(c, cudaGetLastError(), "k_csr_rows")) != XT_OK) break;
    if ((s = check_err(c, "csr")) != XT_OK) break;
    if (!canonical) {
      s = build_from_edges(c, nv, ne_in, rows, t32, orient, g);
      if (s == XT_OK) g->n_input = ne_in;
      break;
    }
    if (orient != XT_ORIENT_ID && orient != XT_ORIENT_DEGREE) {
      s = set_error(c, XT_ERR_INVALID, "bad orientation");
      break;
    }
    g->ctx = c;
    g->nv = nv;
    g->n_input = ne_in;
    g->orient = orient;
    const int b = bits_for(nv);
    uint64_t *keys = nullptr, *sel = nullptr;
    uint8_t *flags = nullptr;
    int64_t m = 0;
    do {
      if ((s = dalloc_n(c, &keys, n1)) != XT_OK) break;
      if ((s = dalloc_n(c, &sel, n1)) != XT_OK) break;
      if ((s = dalloc_n(c, &flags, n1)) != XT_OK) break;
      if ((s = dalloc_n(c, &g->d_deg, size_t(nv))) != XT_OK) break;
      k_degree_from_off<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(d_off, nv, g->d_deg);
      if (ne_in > 0) {
        k_csr_orient_keys<<<counted(c, grid_for(ne_in, B, c->sm_count)), B, 0, c->stream>>>(rows, t32, ne_in, d_off, orient, b,
                                                                               keys, flags);
        if ((s = cuda_status(c, cudaGetLastError(), "k_csr_orient_keys")) != XT_OK) break;
        if ((s = select_flagged(c, keys, flags, sel, ne_in, &m)) != XT_OK) break;
      }
      s = finish_graph(c, sel, m, nv, b, g);
    } while (0);
    dfree(c, keys);
    dfree(c, sel);
    dfree(c, flags);
    if (s != XT_OK) free_graph_device(g);
  } while (0);
  dfree(c, rows);
  dfree(c, t32);
  return s;
}

void free_graph_device(Graph *g) {
  if (!g->ctx) return;
  free_plan(g);
  dfree(g->ctx, g->d_off);
  dfree(g->ctx, g->d_col);
  dfree(g->ctx, g->d_ioff);
  dfree(g->ctx, g->d_icol);
  dfree(g->ctx, g->d_deg);
  g->d_off = nullptr;
  g->d_col = nullptr;
  g->d_ioff = nullptr;
  g->d_icol = nullptr;
  g->d_deg = nullptr;
}

}  // namespace xt
