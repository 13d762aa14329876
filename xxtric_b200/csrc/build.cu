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
#include <vector>

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

// (lo[i], hi[i]) = (min, max) of row i's ends; self loops keep lo == hi and
// are dropped later. With deg != null, every non-loop row also counts one
// for each end: the degree with repeated rows counted again, which orders
// the vertices as well as the true degree does (any total order gives the
// same triangle count).
__global__ void k_edge_keys(const int32_t *__restrict__ src, const int32_t *__restrict__ dst, int64_t ne,
                            int64_t nv, uint32_t *__restrict__ lo, uint32_t *__restrict__ hi,
                            int32_t *__restrict__ deg, int *__restrict__ err) {
  XT_GRID_STRIDE(i, ne) {
    int64_t s = src[i], d = dst[i];
    if (s < 0 || d < 0 || s >= nv || d >= nv) {
      atomicOr(err, 1);
      s = 0;
      d = 0;
    }
    const uint32_t l = uint32_t(s < d ? s : d), h = uint32_t(s < d ? d : s);
    lo[i] = l;
    hi[i] = h;
    if (deg && l != h) {
      atomicAdd(&deg[l], 1);
      atomicAdd(&deg[h], 1);
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

// (lo, hi) in input ids -> (row, col) = (low rank, high rank), in place.
// Four rows a thread through 16-byte loads and stores where both arrays
// are 16-byte aligned (then eight table lookups are in flight at once), one
// at a time otherwise and for the last m % 4.
__global__ void k_relabel_split(uint32_t *__restrict__ lo, uint32_t *__restrict__ hi, int64_t m,
                                const int32_t *__restrict__ o2n) {
  const bool vec = ((reinterpret_cast<uintptr_t>(lo) | reinterpret_cast<uintptr_t>(hi)) & 15) == 0;
  const int64_t m4 = vec ? m / 4 : 0;
  XT_GRID_STRIDE(i, m4) {
    const uint4 l = reinterpret_cast<const uint4 *>(lo)[i], h = reinterpret_cast<const uint4 *>(hi)[i];
    const uint32_t a0 = o2n[l.x], a1 = o2n[l.y], a2 = o2n[l.z], a3 = o2n[l.w];
    const uint32_t c0 = o2n[h.x], c1 = o2n[h.y], c2 = o2n[h.z], c3 = o2n[h.w];
    reinterpret_cast<uint4 *>(lo)[i] = make_uint4(min(a0, c0), min(a1, c1), min(a2, c2), min(a3, c3));
    reinterpret_cast<uint4 *>(hi)[i] = make_uint4(max(a0, c0), max(a1, c1), max(a2, c2), max(a3, c3));
  }
  XT_GRID_STRIDE(j, m - 4 * m4) {
    const int64_t i = 4 * m4 + j;
    const uint32_t a = uint32_t(o2n[lo[i]]), c = uint32_t(o2n[hi[i]]);
    lo[i] = a < c ? a : c;
    hi[i] = a < c ? c : a;
  }
}

// ---------------------------------------------------------------------------
// Row buckets. After the rows are sorted by their low end alone, bucket r =
// bk[rstart[r] .. rstart[r + 1]) holds the high ends of row r in input order,
// repeats and self loops (the value r) included. Each bucket is then sorted
// and made unique in place by the tier its length L picks: a thread's
// registers for L <= 16, a warp's registers for L <= 1,024, a CTA's shared
// memory for L <= 32,768, one device radix sort per row above that. ulen[r]
// = the row's unique length; its first ulen[r] entries are the row's
// columns, ascending.

constexpr int kRowThreadMax = 16;
constexpr int kRowWarpMax = 1024;
constexpr int kRowCtaMax = 32768;
constexpr int kRowCtaThreads = 1024;
constexpr uint32_t kNoCol = 0xffffffffu;  // above every column (columns are below 2^31)

// compare-exchange toward ascending (asc) or descending order
__device__ __forceinline__ void cmpx(uint32_t &x, uint32_t &y, bool asc) {
  const uint32_t lo = min(x, y), hi = max(x, y);
  x = asc ? lo : hi;
  y = asc ? hi : lo;
}

// bitonic sorting network over N registers, ascending
template <int N>
__device__ __forceinline__ void net_sort(uint32_t (&v)[N]) {
#pragma unroll
  for (int size = 2; size <= N; size <<= 1)
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1)
#pragma unroll
      for (int i = 0; i < N; i++)
        if ((i & stride) == 0) cmpx(v[i], v[i | stride], (i & size) == 0);
}

// one row of L <= N entries in a thread's registers: sort, drop repeats and
// the self loop, write back in place
template <int N>
__device__ __forceinline__ int64_t thread_row(uint32_t *__restrict__ bk, int64_t a, int L, uint32_t r) {
  uint32_t v[N];
#pragma unroll
  for (int j = 0; j < N; j++) v[j] = j < L ? bk[a + j] : kNoCol;
  net_sort<N>(v);
  int64_t q = 0;
  uint32_t prev = kNoCol;
#pragma unroll
  for (int j = 0; j < N; j++) {
    if (j < L && v[j] != prev && v[j] != r) bk[a + q++] = v[j];
    prev = v[j];
  }
  return q;
}

// The lists of rows the thread tier passes on: the warp tier by K (entries
// per lane: 1, 2, 4, 8, 16, 32), the CTA tier and the device tier. List t
// starts at lists + base[t] and holds cap[t] rows at most (a row of list t
// has more than kListMin[t] entries, so n / (kListMin[t] + 1) + 1 bound it).
constexpr int kLists = 8;
constexpr int64_t kListMin[kLists] = {16, 32, 64, 128, 256, 512, kRowWarpMax, kRowCtaMax};
struct RowLists {
  int64_t base[kLists];
};

__device__ __forceinline__ int row_list(int64_t L) {
  if (L <= kRowThreadMax) return -1;
  if (L <= kRowWarpMax) {
    int t = 0;
    while (L > (int64_t(32) << t)) t++;
    return t;  // K = 1 << t
  }
  return L <= kRowCtaMax ? 6 : 7;
}

// Every row with L <= kRowThreadMax, a thread each; longer rows go to their
// list (warp-aggregated appends; nl[t] counts list t, nl[kLists] takes the
// longest row of the CTA list). A warp takes 32 consecutive rows.
__global__ void k_rows_thread(const int64_t *__restrict__ rstart, int64_t nv, uint32_t *__restrict__ bk,
                              int64_t *__restrict__ ulen, int32_t *__restrict__ lists, RowLists rl,
                              unsigned long long *__restrict__ nl) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t base = w0 * 32; base < nv; base += nw * 32) {
    const int64_t r = base + lane;
    const bool in = r < nv;
    const int64_t a = in ? rstart[r] : 0, L = in ? rstart[r + 1] - a : 0;
    if (in && L <= kRowThreadMax) {
      int64_t q;
      if (L <= 1) q = (L == 1 && bk[a] != uint32_t(r)) ? 1 : 0;
      else if (L <= 4) q = thread_row<4>(bk, a, int(L), uint32_t(r));
      else if (L <= 8) q = thread_row<8>(bk, a, int(L), uint32_t(r));
      else q = thread_row<16>(bk, a, int(L), uint32_t(r));
      ulen[r] = q;
    }
    const int tier = in ? row_list(L) : -1;
    const unsigned any = __ballot_sync(0xffffffffu, tier >= 0);
    if (!any) continue;
    if (tier == 6) atomicMax(&nl[kLists], (unsigned long long)L);
#pragma unroll
    for (int t = 0; t < kLists; t++) {
      const unsigned m = __ballot_sync(0xffffffffu, tier == t);
      if (!m) continue;
      const int leader = __ffs(m) - 1;
      unsigned long long at = 0;
      if (lane == leader) at = atomicAdd(&nl[t], (unsigned long long)__popc(m));
      at = __shfl_sync(0xffffffffu, at, leader);
      if (tier == t) lists[rl.base[t] + int64_t(at) + __popc(m & ((1u << lane) - 1u))] = int32_t(r);
    }
  }
}

// One row of 32 K entries at most in a warp's registers, striped (entry e =
// k * 32 + lane in v[k], so loads and stores coalesce): bitonic sort (pairs
// at distance below 32 across lanes by shuffle, farther ones inside a lane),
// then the unique entries compacted in place by ballot.
template <int K>
__device__ __forceinline__ void warp_row(uint32_t *__restrict__ bk, int64_t a, int L, uint32_t r,
                                         int64_t *__restrict__ ulen_r, int lane) {
  uint32_t v[K];
#pragma unroll
  for (int k = 0; k < K; k++) v[k] = k * 32 + lane < L ? bk[a + k * 32 + lane] : kNoCol;
#pragma unroll
  for (int size = 2; size <= 32 * K; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      if (stride >= 32) {
        const int ks = stride >> 5;
#pragma unroll
        for (int k = 0; k < K; k++)
          if ((k & ks) == 0) cmpx(v[k], v[k | ks], ((k * 32) & size) == 0);
      } else {
        const bool lower = (lane & stride) == 0;
#pragma unroll
        for (int k = 0; k < K; k++) {
          const uint32_t o = __shfl_xor_sync(0xffffffffu, v[k], stride);
          const bool asc = ((k * 32 + lane) & size) == 0;
          v[k] = (lower == asc) ? min(v[k], o) : max(v[k], o);
        }
      }
    }
  }
  int64_t q = 0;
  uint32_t last = kNoCol;  // the entry before this k's lane 0
  const unsigned below = (1u << lane) - 1u;
#pragma unroll
  for (int k = 0; k < K; k++) {
    uint32_t p = __shfl_up_sync(0xffffffffu, v[k], 1);
    if (lane == 0) p = last;
    const bool uq = k * 32 + lane < L && v[k] != p && v[k] != r;
    const unsigned m = __ballot_sync(0xffffffffu, uq);
    if (uq) bk[a + q + __popc(m & below)] = v[k];
    q += __popc(m);
    last = __shfl_sync(0xffffffffu, v[k], 31);
  }
  if (lane == 0) *ulen_r = q;
}

// warp list K: a warp per row
template <int K>
__global__ void k_rows_warp(const int32_t *__restrict__ list, const unsigned long long *__restrict__ n,
                            const int64_t *__restrict__ rstart, uint32_t *__restrict__ bk,
                            int64_t *__restrict__ ulen) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  const int64_t cnt = int64_t(*n);
  for (int64_t i = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; i < cnt; i += nw) {
    const int32_t r = list[i];
    const int64_t a = rstart[r];
    warp_row<K>(bk, a, int(rstart[r + 1] - a), uint32_t(r), &ulen[r], lane);
  }
}

// A sorted row of L entries (src) -> its unique entries without the self
// loop, compacted into dst, which may be src itself: a chunk's entries are
// all read before the scan's barrier, and an entry moves only down, so no
// write reaches an entry a later chunk still reads. All T threads of the
// CTA call it; returns the unique length.
template <int T>
__device__ int64_t cta_unique(const uint32_t *src, int64_t L, uint32_t r, uint32_t *dst) {
  using Scan = cub::BlockScan<int, T>;
  __shared__ typename Scan::TempStorage ts;
  int64_t q = 0;
  for (int64_t c0 = 0; c0 < L; c0 += T) {
    const int64_t e = c0 + threadIdx.x;
    const uint32_t x = e < L ? src[e] : kNoCol;
    const uint32_t p = (e > 0 && e < L) ? src[e - 1] : kNoCol;
    const int uq = (e < L && x != p && x != r) ? 1 : 0;
    int pos, tot;
    Scan(ts).ExclusiveSum(uq, pos, tot);
    if (uq) dst[q + pos] = x;
    q += tot;
    __syncthreads();  // ts is reused by the next chunk
  }
  return q;
}

// Bitonic stages on a 1,024-entry chunk in a warp's registers, striped
// (entry k * 32 + lane in v[k]): chunk_presort runs the network's sizes 2 to
// 512 (directions from the entry's place in the chunk); chunk_merge runs the
// strides 512 to 1 of one larger size, whose direction (asc) is the same
// for the whole chunk.
__device__ __forceinline__ void chunk_presort(uint32_t (&v)[32], int lane) {
#pragma unroll
  for (int size = 2; size <= 512; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      if (stride >= 32) {
        const int ks = stride >> 5;
#pragma unroll
        for (int k = 0; k < 32; k++)
          if ((k & ks) == 0) cmpx(v[k], v[k | ks], ((k * 32) & size) == 0);
      } else {
        const bool lower = (lane & stride) == 0;
#pragma unroll
        for (int k = 0; k < 32; k++) {
          const uint32_t o = __shfl_xor_sync(0xffffffffu, v[k], stride);
          const bool asc = ((k * 32 + lane) & size) == 0;
          v[k] = (lower == asc) ? min(v[k], o) : max(v[k], o);
        }
      }
    }
  }
}
__device__ __forceinline__ void chunk_merge(uint32_t (&v)[32], int lane, bool asc) {
#pragma unroll
  for (int ks = 16; ks > 0; ks >>= 1)
#pragma unroll
    for (int k = 0; k < 32; k++)
      if ((k & ks) == 0) cmpx(v[k], v[k | ks], asc);
#pragma unroll
  for (int stride = 16; stride > 0; stride >>= 1) {
    const bool lower = (lane & stride) == 0;
#pragma unroll
    for (int k = 0; k < 32; k++) {
      const uint32_t o = __shfl_xor_sync(0xffffffffu, v[k], stride);
      v[k] = (lower == asc) ? min(v[k], o) : max(v[k], o);
    }
  }
}

// The CTA list: a CTA per row, N = the power of two at or above L (2,048 to
// kRowCtaMax) entries in shared memory (the launch gives as many as the
// list's longest row needs). Each warp sorts 1,024-entry chunks in
// registers (the network's sizes up to 1,024); each larger size then runs
// its strides of 1,024 and up in shared memory and the rest chunk by chunk
// in registers again.
constexpr int kCtaSortThreads = 512;
__global__ void __launch_bounds__(kCtaSortThreads) k_rows_cta(const int32_t *__restrict__ list,
                                                              const unsigned long long *__restrict__ n,
                                                              const int64_t *__restrict__ rstart,
                                                              uint32_t *__restrict__ bk, int64_t *__restrict__ ulen) {
  extern __shared__ uint32_t srow[];
  constexpr int W = kCtaSortThreads / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t cnt = int64_t(*n);
  for (int64_t i = blockIdx.x; i < cnt; i += gridDim.x) {
    const int32_t r = list[i];
    const int64_t a = rstart[r];
    const int L = int(rstart[r + 1] - a);
    int N = 2048;
    while (N < L) N <<= 1;
    const int nc = N >> 10;
    for (int c = warp; c < nc; c += W) {
      uint32_t v[32];
#pragma unroll
      for (int k = 0; k < 32; k++) {
        const int e = (c << 10) + k * 32 + lane;
        v[k] = e < L ? bk[a + e] : kNoCol;
      }
      chunk_presort(v, lane);
      chunk_merge(v, lane, (c & 1) == 0);
#pragma unroll
      for (int k = 0; k < 32; k++) srow[(c << 10) + k * 32 + lane] = v[k];
    }
    __syncthreads();
    for (int size = 2048; size <= N; size <<= 1) {
      for (int stride = size >> 1; stride >= 1024; stride >>= 1) {
        for (int j = threadIdx.x; j < N / 2; j += kCtaSortThreads) {
          const int x = ((j & ~(stride - 1)) << 1) | (j & (stride - 1)), y = x + stride;
          uint32_t u = srow[x], w = srow[y];
          cmpx(u, w, (x & size) == 0);
          srow[x] = u;
          srow[y] = w;
        }
        __syncthreads();
      }
      for (int c = warp; c < nc; c += W) {
        uint32_t v[32];
#pragma unroll
        for (int k = 0; k < 32; k++) v[k] = srow[(c << 10) + k * 32 + lane];
        chunk_merge(v, lane, ((c << 10) & size) == 0);
#pragma unroll
        for (int k = 0; k < 32; k++) srow[(c << 10) + k * 32 + lane] = v[k];
      }
      __syncthreads();
    }
    const int64_t q = cta_unique<kCtaSortThreads>(srow, L, uint32_t(r), bk + a);
    if (threadIdx.x == 0) ulen[r] = q;
    __syncthreads();  // srow is refilled by the next row
  }
}

// the device list's {row, start, length} into spans (4 fields a row; the
// host adds the fourth)
__global__ void k_rows_spans(const int32_t *__restrict__ list, int64_t nd, const int64_t *__restrict__ rstart,
                             int64_t *__restrict__ spans) {
  XT_GRID_STRIDE(i, nd) {
    const int32_t r = list[i];
    spans[4 * i] = r;
    spans[4 * i + 1] = rstart[r];
    spans[4 * i + 2] = rstart[r + 1] - rstart[r];
  }
}

// The device list's rows (spans[i] = {row, start, length, offset}, offset =
// the entries of the rows before it) into one key array, (i << 32 | column),
// so a single device radix sort orders every row at once; back again after
// it.
__global__ void k_rows_gather(const int64_t *__restrict__ spans, int64_t nd, const uint32_t *__restrict__ bk,
                              uint64_t *__restrict__ keys) {
  for (int64_t i = blockIdx.x; i < nd; i += gridDim.x) {
    const int64_t a = spans[4 * i + 1], L = spans[4 * i + 2], o = spans[4 * i + 3];
    for (int64_t j = threadIdx.x; j < L; j += blockDim.x) keys[o + j] = (uint64_t(i) << 32) | bk[a + j];
  }
}
__global__ void __launch_bounds__(kRowCtaThreads) k_rows_scatter_unique(const int64_t *__restrict__ spans,
                                                                        int64_t nd, const uint64_t *__restrict__ keys,
                                                                        uint32_t *bk, int64_t *__restrict__ ulen) {
  for (int64_t i = blockIdx.x; i < nd; i += gridDim.x) {
    const int64_t r = spans[4 * i], a = spans[4 * i + 1], L = spans[4 * i + 2], o = spans[4 * i + 3];
    for (int64_t j = threadIdx.x; j < L; j += blockDim.x) bk[a + j] = uint32_t(keys[o + j]);
    __syncthreads();
    const int64_t q = cta_unique<kRowCtaThreads>(bk + a, L, uint32_t(r), bk + a);
    if (threadIdx.x == 0) ulen[r] = q;
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

// Unique rows -> the out-CSR and the unsorted in-records. A warp takes 32
// consecutive rows, whose padded spans are contiguous in colp (and their
// columns in col): it walks those spans 32 entries at a time, each lane
// finding its entry's row among the 32 by a binary search over the rows'
// padded starts, held one per lane, so the writes coalesce however short the
// rows are. Entry t of row u is column v = bk[rstart[u] + t] while t <
// ulen[u] (kPadSentinel after it); its out-CSR position p = off[u] + t also
// gets the in-record of edge u->v (the suffix after t: colp[poff[u] + t + 1,
// poff[u] + ulen[u])) and its sort key, v << lb | the suffix length's class
// (lb of its 7 bits, as many as fit beside v in 31 bits).
__global__ void k_rows_emit(const int64_t *__restrict__ rstart, const uint32_t *__restrict__ bk, int64_t nv, int lb,
                            const int64_t *__restrict__ off, const int64_t *__restrict__ poff,
                            int32_t *__restrict__ col, int32_t *__restrict__ colp, uint32_t *__restrict__ ik,
                            InRec *__restrict__ rec) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t base = w0 * 32; base < nv; base += nw * 32) {
    const int64_t r = base + lane, rc = r < nv ? r : nv;  // lanes past nv: empty rows at the end
    const int64_t o = off[rc], len = off[r < nv ? r + 1 : nv] - o, p = poff[rc];
    const int64_t a = r < nv ? rstart[r] : 0;
    const int64_t p0 = __shfl_sync(0xffffffffu, p, 0);
    const int64_t pend = poff[base + 32 < nv ? base + 32 : nv];
    for (int64_t q0 = p0; q0 < pend; q0 += 32) {
      const int64_t q = q0 + lane;
      int j = 0;  // the last row starting at or before q
#pragma unroll
      for (int step = 16; step; step >>= 1)
        if (__shfl_sync(0xffffffffu, p, j + step) <= q) j += step;
      const int64_t pj = __shfl_sync(0xffffffffu, p, j), lj = __shfl_sync(0xffffffffu, len, j);
      const int64_t oj = __shfl_sync(0xffffffffu, o, j), aj = __shfl_sync(0xffffffffu, a, j);
      if (q < pend) {
        const int64_t t = q - pj;
        if (t < lj) {
          const uint32_t x = bk[aj + t];
          const int64_t sl = lj - t - 1;
          col[oj + t] = int32_t(x);
          colp[q] = int32_t(x);
          ik[oj + t] = (x << lb) | (lb > 0 ? len_class_desc(sl) >> (7 - lb) : 0u);
          rec[oj + t] = make_inrec(q + 1, sl);
        } else {
          colp[q] = kPadSentinel;
        }
      }
    }
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
    recp[p] = make_inrec(poff[u] + (p - a) + 1, len);  // the suffix, in the padded column array
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
// (internal -> input id) and relabels n rows in place: packed keys (lo << b
// | hi, input ids) to (low rank << b | high rank), or, with keys == null,
// the split ends lo[] / hi[] to (low rank, high rank). The rank is a stable
// sort of the ids keyed by degree alone (the ids enter in ascending order,
// so ties keep id order), on as many key bits as the largest degree needs.
static xt_status rank_and_relabel(Ctx *c, int32_t *deg, int64_t nv, int b, uint64_t *keys, int64_t n, Graph *g,
                                  uint32_t *lo = nullptr, uint32_t *hi = nullptr) {
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
    if (n > 0 && keys) k_relabel_edges<<<counted(c, grid_for(n, B, c->sm_count)), B, 0, c->stream>>>(keys, n, b, o2n);
    if (n > 0 && !keys) k_relabel_split<<<counted(c, grid_for(n, B, c->sm_count)), B, 0, c->stream>>>(lo, hi, n, o2n);
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
  xt_status s = dalloc_n(c, &r0, size_t(m) + 2);
  if (s == XT_OK) s = dalloc_n(c, &r1, size_t(m) + 2);
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
    if (total >= kMaxColp) return set_error(c, XT_ERR_OVERFLOW, "2^35 or more padded columns: beyond what the in-records address");
    XT_TRY(dalloc_n(c, &g->d_colp, size_t(total > 0 ? total : 8)));
    g->colp_len = total;
    if (total > 0)
      k_pad_fill<<<counted(c, grid_for(m, B, c->sm_count)), B, 0, c->stream>>>(keys, m, b, g->d_off, g->d_poff,
                                                                               g->d_colp);
    XT_CUDA(c, cudaGetLastError());
  }
  XT_TRY(dalloc_n(c, &g->d_ioff, size_t(nv + 1)));
  if (m == 0) {
    XT_TRY(dalloc_n(c, &g->d_irec, 2));
    XT_CUDA(c, cudaMemsetAsync(g->d_ioff, 0, sizeof(int64_t) * (nv + 1), c->stream));
    return XT_OK;
  }
  return build_in_records(c, keys, spare, m, nv, b, g);
}

// The out-CSR and the in-records from n rows grouped by their low end:
// rows_s (the low ends, ascending) and cols_s (the high ends, in any order
// within a row; repeats and self loops allowed). kbuf: n 8-byte entries
// disjoint from cols_s, which take the in-record sort's keys (both of its
// buffers).
static xt_status rows_to_csr(Ctx *c, const uint32_t *rows_s, uint32_t *cols_s, int64_t n, int64_t nv, int b,
                             uint64_t *kbuf, Graph *g) {
  const int B = 256;
  int64_t *rstart = nullptr, *ulen = nullptr, *spans = nullptr;
  int32_t *lists = nullptr;
  unsigned long long *nl = nullptr;
  uint64_t *hk = nullptr;
  InRec *r0 = nullptr, *r1 = nullptr;
  void *tmp = nullptr;
  xt_status s = XT_OK;
  do {
    // bucket bounds: the runs of the sorted low ends
    if ((s = dalloc_n(c, &rstart, size_t(nv + 1))) != XT_OK) break;
    if ((s = keys_to_csr<uint32_t>(c, rows_s, n, nv, 0, rstart, nullptr)) != XT_OK) break;
    if ((s = dalloc_n(c, &ulen, size_t(nv + 1))) != XT_OK) break;
    RowLists rl;
    int64_t ltot = 0;
    for (int t = 0; t < kLists; t++) {
      rl.base[t] = ltot;
      ltot += n / (kListMin[t] + 1) + 1;
    }
    if ((s = dalloc_n(c, &lists, size_t(ltot))) != XT_OK) break;
    if ((s = dalloc_n(c, &nl, kLists + 1)) != XT_OK) break;
    if ((s = cuda_status(c, cudaMemsetAsync(nl, 0, (kLists + 1) * sizeof(*nl), c->stream), "memset")) != XT_OK) break;
    if ((s = cuda_status(c, cudaMemsetAsync(ulen + nv, 0, sizeof(int64_t), c->stream), "memset")) != XT_OK) break;
    // each bucket sorted and made unique in place by its tier
    k_rows_thread<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(rstart, nv, cols_s, ulen, lists, rl,
                                                                                 nl);
    if ((s = cuda_status(c, cudaGetLastError(), "row sort")) != XT_OK) break;
    unsigned long long hn[kLists + 1];
    if ((s = cuda_status(c, cudaMemcpyAsync(hn, nl, sizeof(hn), cudaMemcpyDeviceToHost, c->stream), "D2H")) != XT_OK)
      break;
    if ((s = cuda_status(c, cudaStreamSynchronize(c->stream), "sync")) != XT_OK) break;
    using WarpFn = void (*)(const int32_t *, const unsigned long long *, const int64_t *, uint32_t *, int64_t *);
    const WarpFn wfn[6] = {k_rows_warp<1>, k_rows_warp<2>, k_rows_warp<4>,
                           k_rows_warp<8>, k_rows_warp<16>, k_rows_warp<32>};
    for (int t = 0; t < 6 && s == XT_OK; t++) {
      if (!hn[t]) continue;
      const int64_t blocks = std::min<int64_t>((int64_t(hn[t]) + 7) / 8, int64_t(c->sm_count) * 16);
      wfn[t]<<<counted(c, dim3(unsigned(blocks))), B, 0, c->stream>>>(lists + rl.base[t], nl + t, rstart, cols_s,
                                                                      ulen);
      s = cuda_status(c, cudaGetLastError(), "row sort");
    }
    if (s != XT_OK) break;
    if (hn[6]) {
      int N = 2048;
      while (uint64_t(N) < hn[kLists]) N <<= 1;
      const int smem = N * int(sizeof(uint32_t));
      if ((s = cuda_status(c, cudaFuncSetAttribute(k_rows_cta, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                           "attr")) != XT_OK)
        break;
      const int64_t blocks = std::min<int64_t>(int64_t(hn[6]), int64_t(c->sm_count) * 4);
      k_rows_cta<<<counted(c, dim3(unsigned(blocks))), kCtaSortThreads, smem, c->stream>>>(
          lists + rl.base[6], nl + 6, rstart, cols_s, ulen);
      if ((s = cuda_status(c, cudaGetLastError(), "row sort")) != XT_OK) break;
    }
    const int64_t nd = int64_t(hn[7]);
    if (nd > 0) {  // rows above kRowCtaMax entries: one device radix sort of them all
      std::vector<int64_t> h(4 * nd);
      if ((s = dalloc_n(c, &spans, size_t(4 * nd))) != XT_OK) break;
      k_rows_spans<<<counted(c, grid_for(nd, B, c->sm_count)), B, 0, c->stream>>>(lists + rl.base[7], nd, rstart,
                                                                                 spans);
      if ((s = cuda_status(c, cudaMemcpyAsync(h.data(), spans, sizeof(int64_t) * 4 * nd, cudaMemcpyDeviceToHost,
                                              c->stream), "D2H")) != XT_OK)
        break;
      if ((s = cuda_status(c, cudaStreamSynchronize(c->stream), "sync")) != XT_OK) break;
      int64_t H = 0;
      for (int64_t i = 0; i < nd; i++) {
        h[4 * i + 3] = H;
        H += h[4 * i + 2];
      }
      if ((s = cuda_status(c, cudaMemcpyAsync(spans, h.data(), sizeof(int64_t) * 4 * nd, cudaMemcpyHostToDevice,
                                              c->stream), "H2D")) != XT_OK)
        break;
      if ((s = dalloc_n(c, &hk, size_t(2 * H))) != XT_OK) break;
      const unsigned gb = unsigned(std::min<int64_t>(nd, int64_t(c->sm_count) * 4));
      k_rows_gather<<<counted(c, dim3(gb)), B, 0, c->stream>>>(spans, nd, cols_s, hk);
      if ((s = cuda_status(c, cudaGetLastError(), "row gather")) != XT_OK) break;
      int ib = 1;
      while ((int64_t(1) << ib) < nd) ib++;
      cub::DoubleBuffer<uint64_t> db(hk, hk + H);
      size_t bytes = 0;
      if ((s = cuda_status(c, cub::DeviceRadixSort::SortKeys(nullptr, bytes, db, H, 0, 32 + ib, c->stream),
                           "row radix sort")) != XT_OK)
        break;
      if ((s = dalloc(c, &tmp, bytes)) != XT_OK) break;
      if ((s = cuda_status(c, cub::DeviceRadixSort::SortKeys(tmp, bytes, db, H, 0, 32 + ib, c->stream),
                           "row radix sort")) != XT_OK)
        break;
      k_rows_scatter_unique<<<counted(c, dim3(gb)), kRowCtaThreads, 0, c->stream>>>(spans, nd, db.Current(), cols_s,
                                                                                     ulen);
      if ((s = cuda_status(c, cudaGetLastError(), "row unique")) != XT_OK) break;
    }
    // offsets of the unique rows, then the padded offsets
    if ((s = dalloc_n(c, &g->d_off, size_t(nv + 1))) != XT_OK) break;
    if ((s = exclusive_scan_i64(c, ulen, g->d_off, nv + 1)) != XT_OK) break;
    int64_t m = 0;
    if ((s = cuda_status(c, cudaMemcpyAsync(&m, g->d_off + nv, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream),
                         "D2H")) != XT_OK)
      break;
    if ((s = cuda_status(c, cudaStreamSynchronize(c->stream), "sync")) != XT_OK) break;
    g->ne = m;
    // Columns are read as aligned 32-byte pairs: pad so the last pair of the
    // last row stays inside the allocation.
    if ((s = dalloc_n(c, &g->d_col, size_t(m) + kColPad)) != XT_OK) break;
    if ((s = cuda_status(c, cudaMemsetAsync(g->d_col + m, 0xff, sizeof(int32_t) * kColPad, c->stream), "memset")) !=
        XT_OK)
      break;
    int64_t *plen = ulen;  // the unique lengths live on in d_off
    if ((s = dalloc_n(c, &g->d_poff, size_t(nv + 1))) != XT_OK) break;
    k_pad_len<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(g->d_off, nv, plen);
    if ((s = cuda_status(c, cudaMemsetAsync(plen + nv, 0, sizeof(int64_t), c->stream), "memset")) != XT_OK) break;
    if ((s = exclusive_scan_i64(c, plen, g->d_poff, nv + 1)) != XT_OK) break;
    int64_t total = 0;
    if ((s = cuda_status(c, cudaMemcpyAsync(&total, g->d_poff + nv, sizeof(int64_t), cudaMemcpyDeviceToHost,
                                            c->stream), "D2H")) != XT_OK)
      break;
    if ((s = cuda_status(c, cudaStreamSynchronize(c->stream), "sync")) != XT_OK) break;
    if (total >= kMaxColp) {
      s = set_error(c, XT_ERR_OVERFLOW, "2^35 or more padded columns: beyond what the in-records address");
      break;
    }
    if ((s = dalloc_n(c, &g->d_colp, size_t(total > 0 ? total : 8))) != XT_OK) break;
    g->colp_len = total;
    if ((s = dalloc_n(c, &g->d_ioff, size_t(nv + 1))) != XT_OK) break;
    if (m == 0) {
      if ((s = dalloc_n(c, &g->d_irec, 2)) != XT_OK) break;
      s = cuda_status(c, cudaMemsetAsync(g->d_ioff, 0, sizeof(int64_t) * (nv + 1), c->stream), "memset");
      break;
    }
    // the out-CSR, with the in-records in position order and their sort keys
    // (head << lb | class, in kbuf), sorted by head and then class (stable:
    // records of one (head, class) stay in position order)
    const int lb = b + 7 <= 31 ? 7 : 31 - b;
    uint32_t *kin = reinterpret_cast<uint32_t *>(kbuf), *kalt = kin + m;
    if ((s = dalloc_n(c, &r0, size_t(m) + 2)) != XT_OK) break;
    if ((s = dalloc_n(c, &r1, size_t(m) + 2)) != XT_OK) break;
    k_rows_emit<<<counted(c, grid_for(nv, B, c->sm_count)), B, 0, c->stream>>>(rstart, cols_s, nv, lb, g->d_off,
                                                                               g->d_poff, g->d_col, g->d_colp, kin, r0);
    if ((s = cuda_status(c, cudaGetLastError(), "row emit")) != XT_OK) break;
    uint32_t *ks = nullptr;
    InRec *rs = nullptr;
    if ((s = sort_pairs_db<InRec>(c, kin, kalt, r0, r1, m, b + lb, &ks, &rs)) != XT_OK) break;
    if ((s = keys_to_csr<uint32_t>(c, ks, m, nv, lb, g->d_ioff, nullptr)) != XT_OK) break;
    g->d_irec = rs;
    if (rs == r0) r0 = nullptr;
    else r1 = nullptr;
  } while (0);
  dfree(c, rstart);
  dfree(c, ulen);
  dfree(c, spans);
  dfree(c, lists);
  dfree(c, nl);
  dfree(c, hk);
  dfree(c, tmp);
  dfree(c, r0);
  dfree(c, r1);
  return s;
}

// Copies the host rows into d_src/d_dst in chunks on the copy stream; the
// context stream turns each chunk into keys (and degree counts) once it has
// landed.
static xt_status upload_and_key(Ctx *c, const HostRows &up, int64_t nv, int64_t ne, int32_t *d_src, int32_t *d_dst,
                                uint32_t *lo, uint32_t *hi, int32_t *deg) {
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
      k_edge_keys<<<counted(c, grid_for(n, B, c->sm_count)), B, 0, c->stream>>>(d_src + a, d_dst + a, n, nv,
                                                                               lo + a, hi + a, deg, c->d_err);
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
  // k0 = the rows' low ends then, from the next 16-byte boundary, their
  // high ends (4 bytes each); k1 = the same for the sort's other buffers
  uint64_t *k0 = nullptr, *k1 = nullptr;
  int32_t *deg = nullptr;
  xt_status s = XT_OK;
  const size_t n1 = size_t(ne > 0 ? ne : 1);
  const int64_t ne4 = (ne + 3) & ~int64_t(3);
  do {
    if ((s = dalloc_n(c, &k0, n1 + 2)) != XT_OK) break;
    if ((s = dalloc_n(c, &k1, n1 + 2)) != XT_OK) break;
    uint32_t *lo = reinterpret_cast<uint32_t *>(k0), *hi = lo + ne4;
    uint32_t *lo2 = reinterpret_cast<uint32_t *>(k1), *hi2 = lo2 + ne4;
    if (orient == XT_ORIENT_DEGREE) {
      if ((s = dalloc_n(c, &deg, size_t(nv))) != XT_OK) break;
      if ((s = cuda_status(c, cudaMemsetAsync(deg, 0, sizeof(int32_t) * nv, c->stream), "memset")) != XT_OK) break;
    }
    if (ne > 0) {
      if (upload) {
        s = upload_and_key(c, *upload, nv, ne, const_cast<int32_t *>(d_src), const_cast<int32_t *>(d_dst), lo, hi,
                           deg);
        if (s != XT_OK) break;
      } else {
        k_edge_keys<<<counted(c, grid_for(ne, B, c->sm_count)), B, 0, c->stream>>>(d_src, d_dst, ne, nv, lo, hi,
                                                                                   deg, c->d_err);
        if ((s = cuda_status(c, cudaGetLastError(), "k_edge_keys")) != XT_OK) break;
      }
      if ((s = check_err(c, "edge list")) != XT_OK) break;
    }
    // rank, then relabel every row in place
    if (orient == XT_ORIENT_DEGREE) {
      if ((s = rank_and_relabel(c, deg, nv, b, nullptr, ne, g, lo, hi)) != XT_OK) break;
      dfree(c, deg);
      deg = nullptr;
    }
    // rows grouped by their low end: a radix sort on the low end's b bits
    uint32_t *rows_s = lo, *cols_s = hi;
    if (ne > 0 && (s = sort_pairs_db<uint32_t>(c, lo, lo2, hi, hi2, ne, b, &rows_s, &cols_s)) != XT_OK) break;
    const bool in_k0 = cols_s == hi;  // the sorted rows are in k0
    s = rows_to_csr(c, rows_s, cols_s, ne, nv, b, in_k0 ? k1 : k0, g);
  } while (0);
  dfree(c, k0);
  dfree(c, k1);
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
  dfree(g->ctx, g->d_irec_u);
  g->d_irec_u = nullptr;
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
