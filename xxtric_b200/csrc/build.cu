// GPU CSR builder: canonicalise (drop self loops, symmetrise, dedup), rank
// the vertices, orient each undirected edge from the lower to the higher rank
// and emit
//   * the oriented out-CSR in rank numbering (int64 offsets, int32 ascending
//     columns), and
//   * per head v, one in-record per edge u->v holding the suffix of N+(u)
//     after v (the candidates w with rank(w) > rank(v)).
//
// Reference behaviour replaced: the reference trusts its input CSR
// (graph.hpp:294-395 reads it verbatim; a duplicated pair over-counts) and
// orients implicitly by vertex id inside the count loop (xxtric.hpp:165-185:
// v = adj(i)[m] > i, then w = adj(i)[n] for n > m). Here the builder makes any
// edge list canonical first, so the count of a canonical input equals the
// reference's count on it; the in-record suffix is exactly the reference's
// n > m range, taken from the head's side.
#include <cub/cub.cuh>

#include <algorithm>

#include "xt_internal.cuh"

namespace xt {

static int bits_for(int64_t n) {
  int b = 1;
  while ((int64_t(1) << b) < n) b++;
  return b;
}

static unsigned grid_for(int64_t n, int block, int sm_count) {
  int64_t g = (n + block - 1) / block;
  int64_t cap = int64_t(sm_count) * 32;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (unsigned)g;
}

#define XT_GRID_STRIDE(i, n) \
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < (n); i += int64_t(gridDim.x) * blockDim.x)

// key = (min << b) | max; self loops keep min == max and are dropped later.
// With deg != null, every non-loop row also counts one for each end: the
// degree with repeated rows counted again, which orders the vertices as well
// as the true degree does (any total order gives the same triangle count).
__global__ void k_edge_keys(const int32_t *__restrict__ src, const int32_t *__restrict__ dst, int64_t ne,
                            int64_t nv, int b, uint64_t *__restrict__ keys, int32_t *__restrict__ deg,
                            int *__restrict__ err) {
  XT_GRID_STRIDE(i, ne) {
    int64_t s = src[i], d = dst[i];
    if (s < 0 || d < 0 || s >= nv || d >= nv) {
      atomicOr(err, 1);
      s = 0;
      d = 0;
    }
    uint64_t lo = uint64_t(s < d ? s : d), hi = uint64_t(s < d ? d : s);
    keys[i] = (lo << b) | hi;
    if (deg && lo != hi) {
      atomicAdd(&deg[lo], 1);
      atomicAdd(&deg[hi], 1);
    }
  }
}

__global__ void k_unique_flags(const uint64_t *__restrict__ keys, int64_t n, int b, uint8_t *__restrict__ flags) {
  const uint64_t mask = (uint64_t(1) << b) - 1;
  XT_GRID_STRIDE(i, n) {
    uint64_t k = keys[i];
    bool first = (i == 0) || (keys[i - 1] != k);
    flags[i] = (first && ((k >> b) != (k & mask))) ? 1 : 0;
  }
}

// every vertex's id (the values of the rank sort, keyed by degree) and the
// largest degree (how many key bits the sort needs)
__global__ void k_rank_ids(const int32_t *__restrict__ deg, int64_t nv, int32_t *__restrict__ ids,
                           unsigned int *__restrict__ dmax) {
  unsigned int mx = 0;
  XT_GRID_STRIDE(x, nv) {
    ids[x] = int32_t(x);
    mx = max(mx, unsigned(deg[x]));
  }
  for (int o = 16; o; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0 && mx) atomicMax(dmax, mx);
}

// ids in (degree, id) order -> input->internal map
__global__ void k_rank_perm(const int32_t *__restrict__ n2o, int64_t nv, int32_t *__restrict__ o2n) {
  XT_GRID_STRIDE(r, nv) o2n[n2o[r]] = int32_t(r);
}

// (lo,hi) in input ids -> (src<<b|dst) in internal ids, src <= dst
__global__ void k_relabel_edges(uint64_t *__restrict__ keys, int64_t m, int b, const int32_t *__restrict__ o2n) {
  const uint64_t mask = (uint64_t(1) << b) - 1;
  XT_GRID_STRIDE(i, m) {
    const uint64_t k = keys[i];
    const uint64_t a = uint64_t(o2n[k >> b]), c = uint64_t(o2n[k & mask]);
    keys[i] = a < c ? ((a << b) | c) : ((c << b) | a);
  }
}

// Sorted keys (row << b | col) -> row lengths and columns. The thread at a
// run's first key adds -start, the one at its last key adds end, so each
// non-empty row ends with end - start (len must start zeroed). The offsets
// are then the exclusive scan of the lengths.
template <class K>
__global__ void k_csr_runs(const K *__restrict__ keys, int64_t m, int b, int64_t *__restrict__ len,
                           int32_t *__restrict__ col) {
  const K mask = (K(1) << b) - 1;
  XT_GRID_STRIDE(i, m) {
    const K k = keys[i];
    const K row = k >> b;
    if (i == 0 || (keys[i - 1] >> b) != row)
      atomicAdd(reinterpret_cast<unsigned long long *>(&len[row]), (unsigned long long)(-i));
    if (i + 1 == m || (keys[i + 1] >> b) != row)
      atomicAdd(reinterpret_cast<unsigned long long *>(&len[row]), (unsigned long long)(i + 1));
    if (col) col[i] = int32_t(k & mask);
  }
}

// row index of every CSR entry (warp per row); optional range checks
__global__ void k_csr_rows(const int64_t *__restrict__ off, int64_t nv, int64_t ne, int32_t *__restrict__ rows,
                           int *__restrict__ err) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t u = warp; u < nv; u += nwarps) {
    int64_t e0 = off[u], e1 = off[u + 1];
    if (e0 < 0 || e1 < e0 || e1 > ne) {
      if (lane == 0 && err) atomicOr(err, 2);
      continue;
    }
    for (int64_t e = e0 + lane; e < e1; e += 32) rows[e] = int32_t(u);
  }
}

__global__ void k_csr_tails32(const int64_t *__restrict__ tails, int64_t n, int64_t nv, int32_t *__restrict__ out,
                              int *__restrict__ err) {
  XT_GRID_STRIDE(i, n) {
    int64_t t = tails[i];
    if (t < 0 || t >= nv) {
      atomicOr(err, 1);
      t = 0;
    }
    out[i] = int32_t(t);
  }
}

// Canonical CSR input check, a warp per row, run once the offsets and ids have
// passed k_csr_rows / k_csr_tails32: every row strictly ascending (no
// repeats), without its own id, and every entry (u,t) listed back in row t
// (binary search of row t, whose bounds were checked). The canonical path
// takes each row's upper part as it stands, so a row out of order would
// reach the count's member sets unsorted and an edge listed from one end
// only would lose its triangles; either sets bit 4 of *err.
__global__ void k_csr_check_canonical(const int64_t *__restrict__ off, const int32_t *__restrict__ t32, int64_t nv,
                                      int *__restrict__ err) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t u = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; u < nv; u += nwarps) {
    const int64_t e0 = off[u], e1 = off[u + 1];
    bool bad = false;
    for (int64_t p = e0 + lane; !bad && p < e1; p += 32) {
      const int32_t t = t32[p];
      bad = t == u || (p > e0 && t32[p - 1] >= t);
      if (!bad) {
        int64_t lo = off[t], hi = off[t + 1];
        const int64_t end = hi;
        while (lo < hi) {
          const int64_t mid = lo + (hi - lo) / 2;
          if (t32[mid] < u) lo = mid + 1;
          else hi = mid;
        }
        bad = lo >= end || t32[lo] != u;
      }
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(err, 4);
  }
}

// canonical CSR input: each undirected edge once, as the entry (u,t), u < t;
// the kept entries stay in (row, column) order
__global__ void k_csr_lower_keys(const int32_t *__restrict__ rows, const int32_t *__restrict__ tails, int64_t n,
                                 int b, uint64_t *__restrict__ keys, uint8_t *__restrict__ flags) {
  XT_GRID_STRIDE(i, n) {
    const int64_t u = rows[i], t = tails[i];
    flags[i] = u < t ? 1 : 0;
    keys[i] = (uint64_t(u) << b) | uint64_t(t);
  }
}

__global__ void k_degree_from_off(const int64_t *__restrict__ off, int64_t nv, int32_t *__restrict__ deg) {
  XT_GRID_STRIDE(i, nv) deg[i] = int32_t(off[i + 1] - off[i]);
}

// padded row lengths: each row rounded up to a multiple of 8 columns
__global__ void k_pad_len(const int64_t *__restrict__ off, int64_t nv, int64_t *__restrict__ plen) {
  XT_GRID_STRIDE(u, nv) plen[u] = (off[u + 1] - off[u] + 7) & ~int64_t(7);
}

// sorted keys (row << b | col) -> the padded columns: key i, the j-th of its
// row, goes to colp[poff[row] + j]; the row's last key also fills the rest
// of the row's padded span with kPadSentinel (a thread per key, so short
// rows cost no idle lanes)
__global__ void k_pad_fill(const uint64_t *__restrict__ keys, int64_t m, int b, const int64_t *__restrict__ off,
                           const int64_t *__restrict__ poff, int32_t *__restrict__ colp) {
  const uint64_t mask = (uint64_t(1) << b) - 1;
  XT_GRID_STRIDE(i, m) {
    const uint64_t k = keys[i];
    const int64_t row = int64_t(k >> b);
    const int64_t q = poff[row] + (i - off[row]);
    colp[q] = int32_t(k & mask);
    if (i + 1 == off[row + 1])
      for (int64_t t = q + 1, e = poff[row + 1]; t < e; t++) colp[t] = kPadSentinel;
  }
}

// Suffix-length class, longest first: 127 - c where c is the length itself
// below 32 and four classes per octave above, so records of one head sort
// into runs of similar length.
__device__ __forceinline__ uint32_t len_class_desc(int64_t len) {
  uint32_t c;
  if (len < 32) {
    c = uint32_t(len);
  } else {
    const int lg = 63 - __clzll(len);
    c = 32u + 4u * uint32_t(lg - 5) + uint32_t((len >> (lg - 2)) & 3);
  }
  return 127u - (c < 127u ? c : 127u);
}

// (head << lb | length class) sort key for every out-CSR position, and the
// position's in-record, both written in position order (rows ascend with
// positions, so the row reads are near sequential): lb (0..7) bits of the
// class fit beside the head in 31 bits. The records then travel through the
// sort as its values, so no gather from random positions follows.
__global__ void k_in_keys(const uint64_t *__restrict__ keys, int b, const int64_t *__restrict__ off,
                          const int64_t *__restrict__ poff, int64_t m, int lb, uint32_t *__restrict__ ik,
                          InRec *__restrict__ recp) {
  const uint64_t mask = (uint64_t(1) << b) - 1;
  XT_GRID_STRIDE(p, m) {
    const uint64_t e = keys[p];  // the out-CSR entry at position p: its row and column
    const int32_t u = int32_t(e >> b);
    const int64_t a = off[u], len = off[u + 1] - p - 1;
    uint32_t k = uint32_t(e & mask) << lb;
    if (lb > 0) k |= len_class_desc(len) >> (7 - lb);
    ik[p] = k;
    InRec r;
    r.s = poff[u] + (p - a) + 1;  // the suffix, in the padded column array
    r.len = int32_t(len);
    r.u = u;
    recp[p] = r;
  }
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

// Stable radix sort of (32-bit key, value) pairs on the low end_bit bits,
// ping-ponging between the caller's two buffers of each (no scratch copies of
// the data); *k_sorted / *v_sorted say which buffer holds the result.
template <class V>
static xt_status sort_pairs_db(Ctx *c, uint32_t *k0, uint32_t *k1, V *v0, V *v1, int64_t n, int end_bit,
                               uint32_t **k_sorted, V **v_sorted) {
  cub::DoubleBuffer<uint32_t> dk(k0, k1);
  cub::DoubleBuffer<V> dv(v0, v1);
  size_t bytes = 0;
  XT_CUDA(c, cub::DeviceRadixSort::SortPairs(nullptr, bytes, dk, dv, n, 0, end_bit, c->stream));
  void *tmp = nullptr;
  XT_TRY(dalloc(c, &tmp, bytes));
  cudaError_t e = cub::DeviceRadixSort::SortPairs(tmp, bytes, dk, dv, n, 0, end_bit, c->stream);
  dfree(c, tmp);
  XT_CUDA(c, e);
  *k_sorted = dk.Current();
  *v_sorted = dv.Current();
  return XT_OK;
}

// sorted (row << b | col) keys -> off[nv+1] (and col[m] when col != null)
template <class K>
static xt_status keys_to_csr(Ctx *c, const K *keys, int64_t m, int64_t nv, int b, int64_t *off, int32_t *col) {
  int64_t *len = nullptr;
  XT_TRY(dalloc_n(c, &len, size_t(nv + 1)));
  cudaError_t e = cudaMemsetAsync(len, 0, sizeof(int64_t) * (nv + 1), c->stream);
  if (e == cudaSuccess && m > 0) {
    k_csr_runs<K><<<counted(c, grid_for(m, 256, c->sm_count)), 256, 0, c->stream>>>(keys, m, b, len, col);
    e = cudaGetLastError();
  }
  size_t bytes = 0;
  void *tmp = nullptr;
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, bytes, len, off, nv + 1, c->stream);
  xt_status s = cuda_status(c, e, "csr offsets");
  if (s == XT_OK) s = dalloc(c, &tmp, bytes);
  if (s == XT_OK)
    s = cuda_status(c, cub::DeviceScan::ExclusiveSum(tmp, bytes, len, off, nv + 1, c->stream), "csr offsets");
  dfree(c, tmp);
  dfree(c, len);
  return s;
}

static xt_status exclusive_scan_i64(Ctx *c, const int64_t *in, int64_t *out, int64_t n) {
  size_t bytes = 0;
  XT_CUDA(c, cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, c->stream));
  void *tmp = nullptr;
  XT_TRY(dalloc(c, &tmp, bytes));
  cudaError_t e = cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, n, c->stream);
  dfree(c, tmp);
  XT_CUDA(c, e);
  return XT_OK;
}

static xt_status check_err(Ctx *c, const char *what) {
  int h = 0;
  XT_CUDA(c, cudaMemcpyAsync(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  XT_CUDA(c, cudaStreamSynchronize(c->stream));
  if (h) {
    XT_CUDA(c, cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
    const char *why = (h & 1)   ? ": vertex id outside [0,nv)"
                      : (h & 2) ? ": offsets not monotone in [0,ne]"
                                : ": a row is out of order, repeats an id or holds its own id, or an edge is "
                                  "missing from its other end's row (not a canonical CSR)";
    return set_error(c, XT_ERR_INVALID, std::string(what) + why);
  }
  return XT_OK;
}

// Degree orientation: ranks the vertices by (deg, id) into g->d_perm
// (internal -> input id) and relabels n keys (lo << b | hi, input ids) in
// place to (low rank << b | high rank). The rank is a stable sort of the
// ids keyed by degree alone (the ids enter in ascending order, so ties keep
// id order), on as many key bits as the largest degree needs.
static xt_status rank_and_relabel(Ctx *c, int32_t *deg, int64_t nv, int b, uint64_t *keys, int64_t n, Graph *g) {
  const int B = 256;
  int32_t *ids = nullptr, *o2n = nullptr, *dalt = nullptr;
  unsigned int *d_dmax = nullptr;
  xt_status s = dalloc_n(c, &ids, size_t(nv));
  if (s == XT_OK) s = dalloc_n(c, &dalt, size_t(nv));
  if (s == XT_OK) s = dalloc_n(c, &o2n, size_t(nv));
  if (s == XT_OK) s = dalloc_n(c, &g->d_perm, size_t(nv));
  if (s == XT_OK) s = dalloc_n(c, &d_dmax, 1);
  unsigned int dmax = 0;
  if (s == XT_OK) s = cuda_status(c, cudaMemsetAsync(d_dmax, 0, sizeof(unsigned int), c->stream), "memset");
  if (s == XT_OK) {
    k_rank_ids<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(deg, nv, ids, d_dmax);
    s = cuda_status(c, cudaMemcpyAsync(&dmax, d_dmax, sizeof(unsigned int), cudaMemcpyDeviceToHost, c->stream),
                    "D2H");
  }
  if (s == XT_OK) s = cuda_status(c, cudaStreamSynchronize(c->stream), "sync");
  uint32_t *dk = nullptr;
  int32_t *perm = nullptr;
  if (s == XT_OK) {
    int bits = 1;
    while (bits < 32 && (uint64_t(1) << bits) <= dmax) bits++;
    // keys: the degrees (deg is consumed); values: the ids
    s = sort_pairs_db<int32_t>(c, reinterpret_cast<uint32_t *>(deg), reinterpret_cast<uint32_t *>(dalt), ids,
                               g->d_perm, nv, bits, &dk, &perm);
  }
  if (s == XT_OK && perm != g->d_perm)
    s = cuda_status(c, cudaMemcpyAsync(g->d_perm, perm, sizeof(int32_t) * nv, cudaMemcpyDeviceToDevice, c->stream),
                    "perm");
  if (s == XT_OK) {
    k_rank_perm<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(g->d_perm, nv, o2n);
    if (n > 0) k_relabel_edges<<<counted(c, grid_for(n, B, c->sm_count)), B, 0, c->stream>>>(keys, n, b, o2n);
    s = cuda_status(c, cudaGetLastError(), "relabel");
  }
  dfree(c, ids);
  dfree(c, dalt);
  dfree(c, o2n);
  dfree(c, d_dmax);
  return s;
}

// In-records grouped by head (d_ioff, d_irec), longest suffix first, from the
// out-CSR. keys: the out-CSR's m sorted keys (row << b | col), read here and
// then overwritten; spare: a free buffer of at least m 8-byte entries. The
// 4-byte sort keys of both sides fit in spare; the records are sorted as
// values between two record arrays, one of which becomes d_irec.
static xt_status build_in_records(Ctx *c, uint64_t *keys, uint64_t *spare, int64_t m, int64_t nv, int b, Graph *g) {
  const int B = 256;
  const int lb = b + 7 <= 31 ? 7 : 31 - b;  // key = head << lb | class, 31 bits at most
  uint32_t *kin = reinterpret_cast<uint32_t *>(spare), *kalt = kin + m;
  InRec *r0 = nullptr, *r1 = nullptr;
  xt_status s = dalloc_n(c, &r0, size_t(m));
  if (s == XT_OK) s = dalloc_n(c, &r1, size_t(m));
  if (s == XT_OK) {
    // the sorted keys still hold each position's row and column
    k_in_keys<<<counted(c, grid_for(m, B, c->sm_count)), B, 0, c->stream>>>(keys, b, g->d_off, g->d_poff, m, lb,
                                                                            kin, r0);
    s = cuda_status(c, cudaGetLastError(), "in-keys");
  }
  // stable: records of one (head, class) stay in position order
  uint32_t *ks = nullptr;
  InRec *rs = nullptr;
  if (s == XT_OK) s = sort_pairs_db<InRec>(c, kin, kalt, r0, r1, m, b + lb, &ks, &rs);
  if (s == XT_OK) s = keys_to_csr<uint32_t>(c, ks, m, nv, lb, g->d_ioff, nullptr);
  if (s == XT_OK) {
    g->d_irec = rs;
    dfree(c, rs == r0 ? r1 : r0);
  } else {
    dfree(c, r0);
    dfree(c, r1);
  }
  return s;
}

// keys: m unique oriented edges (src << b | dst, src < dst, internal ids),
// sorted; spare: m more 8-byte entries. Emits the out-CSR and the in-records.
static xt_status finish_csr(Ctx *c, uint64_t *keys, uint64_t *spare, int64_t m, int64_t nv, int b, Graph *g) {
  g->ne = m;
  // Columns are read as aligned 32-byte pairs: pad so the last pair of the
  // last row stays inside the allocation.
  XT_TRY(dalloc_n(c, &g->d_off, size_t(nv + 1)));
  XT_TRY(dalloc_n(c, &g->d_col, size_t(m) + kColPad));
  XT_CUDA(c, cudaMemsetAsync(g->d_col + m, 0xff, sizeof(int32_t) * kColPad, c->stream));
  XT_TRY(keys_to_csr<uint64_t>(c, keys, m, nv, b, g->d_off, g->d_col));
  // padded columns: row starts on 8-column boundaries
  {
    const int B = 256;
    int64_t *plen = nullptr;
    XT_TRY(dalloc_n(c, &g->d_poff, size_t(nv + 1)));
    XT_TRY(dalloc_n(c, &plen, size_t(nv + 1)));
    k_pad_len<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(g->d_off, nv, plen);
    xt_status s = cuda_status(c, cudaMemsetAsync(plen + nv, 0, sizeof(int64_t), c->stream), "memset");
    if (s == XT_OK) s = exclusive_scan_i64(c, plen, g->d_poff, nv + 1);
    int64_t total = 0;
    if (s == XT_OK)
      s = cuda_status(c, cudaMemcpyAsync(&total, g->d_poff + nv, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream),
                      "D2H");
    if (s == XT_OK) s = cuda_status(c, cudaStreamSynchronize(c->stream), "sync");
    dfree(c, plen);
    XT_TRY(s);
    XT_TRY(dalloc_n(c, &g->d_colp, size_t(total > 0 ? total : 8)));
    g->colp_len = total;
    if (total > 0)
      k_pad_fill<<<counted(c, grid_for(m, B, c->sm_count)), B, 0, c->stream>>>(keys, m, b, g->d_off, g->d_poff,
                                                                               g->d_colp);
    XT_CUDA(c, cudaGetLastError());
  }
  XT_TRY(dalloc_n(c, &g->d_ioff, size_t(nv + 1)));
  if (m == 0) {
    XT_TRY(dalloc_n(c, &g->d_irec, 1));
    XT_CUDA(c, cudaMemsetAsync(g->d_ioff, 0, sizeof(int64_t) * (nv + 1), c->stream));
    return XT_OK;
  }
  return build_in_records(c, keys, spare, m, nv, b, g);
}

// Copies the host rows into d_src/d_dst in chunks on the copy stream; the
// context stream turns each chunk into keys (and degree counts) once it has
// landed.
static xt_status upload_and_key(Ctx *c, const HostRows &up, int64_t nv, int64_t ne, int32_t *d_src, int32_t *d_dst,
                                int b, uint64_t *keys, int32_t *deg) {
  constexpr int kChunks = 8;
  const int B = 256;
  if (!c->copy_stream) XT_CUDA(c, cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
  cudaEvent_t ev[kChunks + 1] = {};
  xt_status s = XT_OK;
  for (int i = 0; i <= kChunks && s == XT_OK; i++)
    s = cuda_status(c, cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming), "event");
  // the copy stream starts after the buffers' stream-ordered allocation
  if (s == XT_OK) s = cuda_status(c, cudaEventRecord(ev[kChunks], c->stream), "event");
  if (s == XT_OK) s = cuda_status(c, cudaStreamWaitEvent(c->copy_stream, ev[kChunks], 0), "event");
  const int64_t step = (ne + kChunks - 1) / kChunks;
  for (int i = 0; i < kChunks && s == XT_OK; i++) {
    const int64_t a = int64_t(i) * step, n = std::min(step, ne - a);
    if (n <= 0) break;
    s = cuda_status(c, cudaMemcpyAsync(d_src + a, up.src + a, sizeof(int32_t) * n, cudaMemcpyHostToDevice,
                                       c->copy_stream), "H2D");
    if (s == XT_OK)
      s = cuda_status(c, cudaMemcpyAsync(d_dst + a, up.dst + a, sizeof(int32_t) * n, cudaMemcpyHostToDevice,
                                         c->copy_stream), "H2D");
    if (s == XT_OK) s = cuda_status(c, cudaEventRecord(ev[i], c->copy_stream), "event");
    if (s == XT_OK) s = cuda_status(c, cudaStreamWaitEvent(c->stream, ev[i], 0), "event");
    if (s == XT_OK) {
      k_edge_keys<<<counted(c, grid_for(n, B, c->sm_count)), B, 0, c->stream>>>(d_src + a, d_dst + a, n, nv, b,
                                                                               keys + a, deg, c->d_err);
      s = cuda_status(c, cudaGetLastError(), "k_edge_keys");
    }
  }
  if (s != XT_OK) cudaStreamSynchronize(c->copy_stream);  // no copy outlives a failed build
  // the events have been waited on by the context stream; destroying them now is allowed
  for (int i = 0; i <= kChunks; i++)
    if (ev[i]) cudaEventDestroy(ev[i]);
  return s;
}

xt_status build_from_edges(Ctx *c, int64_t nv, int64_t ne, const int32_t *d_src, const int32_t *d_dst, int orient,
                           Graph *g, const HostRows *upload) {
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
    if (orient == XT_ORIENT_DEGREE) {
      if ((s = dalloc_n(c, &deg, size_t(nv))) != XT_OK) break;
      if ((s = cuda_status(c, cudaMemsetAsync(deg, 0, sizeof(int32_t) * nv, c->stream), "memset")) != XT_OK) break;
    }
    if (ne > 0) {
      if (upload) {
        s = upload_and_key(c, *upload, nv, ne, const_cast<int32_t *>(d_src), const_cast<int32_t *>(d_dst), b, k0,
                           deg);
        if (s != XT_OK) break;
      } else {
        k_edge_keys<<<counted(c, grid_for(ne, B, c->sm_count)), B, 0, c->stream>>>(d_src, d_dst, ne, nv, b, k0,
                                                                                   deg, c->d_err);
        if ((s = cuda_status(c, cudaGetLastError(), "k_edge_keys")) != XT_OK) break;
      }
      if ((s = check_err(c, "edge list")) != XT_OK) break;
    }
    // rank, then relabel every row: one sort of the rows in internal ids
    if (orient == XT_ORIENT_DEGREE) {
      if ((s = rank_and_relabel(c, deg, nv, b, k0, ne, g)) != XT_OK) break;
      dfree(c, deg);
      deg = nullptr;
    }
    if (ne > 0) {
      if ((s = dalloc_n(c, &flags, n1)) != XT_OK) break;
      if ((s = sort_keys(c, k0, k1, ne, 2 * b)) != XT_OK) break;
      k_unique_flags<<<counted(c, grid_for(ne, B, c->sm_count)), B, 0, c->stream>>>(k1, ne, b, flags);
      if ((s = select_flagged(c, k1, flags, k0, ne, &m)) != XT_OK) break;
      dfree(c, flags);
      flags = nullptr;
    }
    // k0[0..m) = unique oriented edges, sorted
    s = finish_csr(c, k0, k1, m, nv, b, g);
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
  if (orient != XT_ORIENT_ID && orient != XT_ORIENT_DEGREE) return set_error(c, XT_ERR_INVALID, "bad orientation");
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
    k_csr_rows<<<counted(c, grid_for(nv * 32, B, c->sm_count)), B, 0, c->stream>>>(d_off, nv, ne_in, rows,
                                                                                   c->d_err);
    k_csr_tails32<<<counted(c, grid_for(ne_in, B, c->sm_count)), B, 0, c->stream>>>(d_tails, ne_in, nv, t32,
                                                                                    c->d_err);
    if ((s = cuda_status(c, cudaGetLastError(), "k_csr_rows")) != XT_OK) break;
    if ((s = check_err(c, "csr")) != XT_OK) break;
    if (canonical) {  // the rows are used as they stand: check the promise first
      k_csr_check_canonical<<<counted(c, grid_for(nv * 32, B, c->sm_count)), B, 0, c->stream>>>(d_off, t32, nv,
                                                                                                c->d_err);
      if ((s = cuda_status(c, cudaGetLastError(), "k_csr_check_canonical")) != XT_OK) break;
      if ((s = check_err(c, "canonical csr")) != XT_OK) break;
    }
    if (!canonical) {
      s = build_from_edges(c, nv, ne_in, rows, t32, orient, g);
      if (s == XT_OK) g->n_input = ne_in;
      break;
    }
    g->ctx = c;
    g->nv = nv;
    g->n_input = ne_in;
    g->orient = orient;
    const int b = bits_for(nv);
    uint64_t *keys = nullptr, *sel = nullptr;
    uint8_t *flags = nullptr;
    int32_t *deg = nullptr;
    int64_t m = 0;
    do {
      if ((s = dalloc_n(c, &keys, n1)) != XT_OK) break;
      if ((s = dalloc_n(c, &sel, n1)) != XT_OK) break;
      if ((s = dalloc_n(c, &flags, n1)) != XT_OK) break;
      if (ne_in > 0) {
        // the u < t entries of sorted symmetric rows: the sorted undirected set
        k_csr_lower_keys<<<counted(c, grid_for(ne_in, B, c->sm_count)), B, 0, c->stream>>>(rows, t32, ne_in, b,
                                                                                           keys, flags);
        if ((s = cuda_status(c, cudaGetLastError(), "k_csr_lower_keys")) != XT_OK) break;
        if ((s = select_flagged(c, keys, flags, sel, ne_in, &m)) != XT_OK) break;
      }
      dfree(c, flags);
      flags = nullptr;
      if (orient == XT_ORIENT_DEGREE) {
        if ((s = dalloc_n(c, &deg, size_t(nv))) != XT_OK) break;
        k_degree_from_off<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(d_off, nv, deg);
        if ((s = rank_and_relabel(c, deg, nv, b, sel, m, g)) != XT_OK) break;
        dfree(c, deg);
        deg = nullptr;
        if (m > 0 && (s = sort_keys(c, sel, keys, m, 2 * b)) != XT_OK) break;
        s = finish_csr(c, keys, sel, m, nv, b, g);
      } else {
        s = finish_csr(c, sel, keys, m, nv, b, g);
      }
    } while (0);
    dfree(c, keys);
    dfree(c, sel);
    dfree(c, flags);
    dfree(c, deg);
    if (s != XT_OK) free_graph_device(g);
  } while (0);
  dfree(c, rows);
  dfree(c, t32);
  return s;
}

void free_graph_device(Graph *g) {
  if (!g->ctx) return;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  g->exec = nullptr;
  dfree(g->ctx, g->d_res);
  g->d_res = nullptr;
  free_plan(g);
  dfree(g->ctx, g->d_off);
  dfree(g->ctx, g->d_col);
  dfree(g->ctx, g->d_ioff);
  dfree(g->ctx, g->d_irec);
  dfree(g->ctx, g->d_colp);
  dfree(g->ctx, g->d_poff);
  dfree(g->ctx, g->d_perm);
  dfree(g->ctx, g->d_group);
  g->d_off = nullptr;
  g->d_col = nullptr;
  g->d_ioff = nullptr;
  g->d_irec = nullptr;
  g->d_colp = nullptr;
  g->d_poff = nullptr;
  g->d_perm = nullptr;
  g->d_group = nullptr;
}

}  // namespace xt
