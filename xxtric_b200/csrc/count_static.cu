// xt_count_device_static: the triangle count of a device CSR in the
// reference's layout (the int64 offsets and tails that single_gpu_count
// takes, counting.cu:537-577) that allocates no device memory at all.
//
// Who needs it: callers that must not allocate on the device while they run,
// e.g. a solver whose device memory is entirely pre-reserved by another
// framework's memory pool, a process that runs under a hard per-process
// memory quota, or a loop that must never take the allocator's lock or
// implicit synchronisation. Those callers pass their inputs and output; every
// scratch word this entry point needs sits in one fixed array in the
// library's module (below), loaded with the module on every GPU that uses the
// library and held until the process exits.
//
// The count uses the reference's vertex-id orientation (u < v < w) straight
// on the symmetric sorted rows, the same membership structures as the main
// count (a bitmap over [min, max] of N+(v), or a hash), and no renumbering.
// Scratch: a header of counters, the split point of every row (the index of
// its first neighbour above the row's own id) and the list of heads whose
// N+(v) needs a whole CTA: 8 bytes per vertex, so at most kMaxNv vertices.
// Each device has its own copy of the array; every call on a device shares
// it and it keeps the previous call's contents, so each call first clears
// the words that must start at zero. Calls whose work overlaps on one device
// (for example, issued on two streams at once) race on it and give wrong
// counts: serialise them.
//
// Input: the entry cannot sort, so it checks the rows first (order, repeats,
// self loops, id range, and that every edge is listed from both ends) and on
// any failure returns XT_ERR_INVALID and leaves *d_count as it was.
//
// Set-up: the first call on a device, with that device current, looks the
// array's device address up (cudaGetSymbolAddress) and keeps it; make that
// first call before any stream capture.
#include <mutex>

#include "xt_internal.cuh"

namespace xt {
namespace nalloc {

constexpr size_t kScratchBytes = (size_t(64) << 20) + 4096;  // 64 MiB + header room
constexpr size_t kHeaderBytes = 256;
constexpr int64_t kMaxNv = int64_t((kScratchBytes - kHeaderBytes) / 8);  // 8 bytes per vertex

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

struct Header {
  unsigned long long triangles;  // the running count
  unsigned long long n_heavy;    // entries of the heavy-head list
  unsigned long long cursor_w;   // next head batch for the warp pass
  unsigned long long cursor_c;   // next heavy head for the CTA pass
  int err;                       // bit 1: an edge lacks its back edge; bit 2: a row fails the row check
};

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kWarpD = 64;          // heads with d+(v) above this go to the CTA pass
constexpr int kWarpWords = 256;     // 256-slot hash or 8192-bit bitmap per warp
constexpr int kBlockPart = 2048;    // members per CTA part
constexpr int kBlockWords = 8192;   // 8192-slot hash or 2^18-bit bitmap per CTA
constexpr int kHeadBatch = 64;      // heads claimed per cursor step in the warp pass
constexpr int32_t kEmpty = -1;

struct Scratch {
  Header *hdr;
  int32_t *split;  // nv: first index in row v whose neighbour is above v
  int32_t *heavy;  // nv: heads for the CTA pass
};

__host__ __device__ inline Scratch carve(unsigned char *base, int64_t nv) {
  Scratch s;
  s.hdr = reinterpret_cast<Header *>(base);
  s.split = reinterpret_cast<int32_t *>(base + kHeaderBytes);
  s.heavy = s.split + nv;
  return s;
}

__global__ void k_na_init(Header *hdr) {
  hdr->triangles = 0;
  hdr->n_heavy = 0;
  hdr->cursor_w = 0;
  hdr->cursor_c = 0;
  hdr->err = 0;
}

// Input check, a warp per row: offsets that are not negative and do not
// decrease, ids in [0, nv), rows strictly ascending (no repeats) and without
// the row's own id. A violation sets hdr->err (bit 2) and the passes below do
// nothing, so an unsorted row or an id past nv cannot steer shared- or
// global-memory indices.
__global__ void k_na_check(int64_t nv, const int64_t *__restrict__ off, const int64_t *__restrict__ tails,
                           Header *hdr) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t v = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; v < nv; v += nwarps) {
    const int64_t e0 = off[v], e1 = off[v + 1];
    bool bad = e0 < 0 || e1 < e0;
    for (int64_t p = e0 + lane; !bad && p < e1; p += 32) {
      const int64_t t = tails[p];
      bad = t < 0 || t >= nv || t == v || (p > e0 && tails[p - 1] >= t);
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(&hdr->err, 2);
  }
}

// Symmetry, a warp per row, once the rows have passed k_na_check: every entry
// t of row v must have v in row t (binary search of the sorted row t). Both
// directions of a missing back edge set hdr->err (bit 1): the count reads
// only the upper parts of the rows and would otherwise drop the triangles
// of an edge listed on one side.
__global__ void k_na_back(int64_t nv, const int64_t *__restrict__ off, const int64_t *__restrict__ tails,
                          Header *hdr) {
  if (hdr->err) return;
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t v = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; v < nv; v += nwarps) {
    bool bad = false;
    for (int64_t p = off[v] + lane; !bad && p < off[v + 1]; p += 32) {
      const int64_t t = tails[p];
      int64_t lo = off[t], hi = off[t + 1];
      while (lo < hi) {
        const int64_t mid = lo + (hi - lo) / 2;
        if (tails[mid] < v) lo = mid + 1;
        else hi = mid;
      }
      bad = lo >= off[t + 1] || tails[lo] != v;
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(&hdr->err, 1);
  }
}

// split point of every row, and the heads whose out-list is too long for a warp
__global__ void k_na_split(int64_t nv, const int64_t *__restrict__ off, const int64_t *__restrict__ tails,
                           Scratch sc) {
  if (sc.hdr->err) return;  // the input check failed
  for (int64_t v = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; v < nv; v += int64_t(gridDim.x) * blockDim.x) {
    int64_t lo = off[v], hi = off[v + 1];
    const int64_t e0 = lo, e1 = hi;
    while (lo < hi) {
      const int64_t mid = lo + (hi - lo) / 2;
      if (tails[mid] <= v) lo = mid + 1;
      else hi = mid;
    }
    sc.split[v] = int32_t(lo - e0);
    const int64_t dplus = e1 - lo, din = lo - e0;
    if (dplus > kWarpD && din > 0) sc.heavy[atomicAdd(&sc.hdr->n_heavy, 1ull)] = int32_t(v);
  }
}

__device__ __forceinline__ uint32_t na_hash(int32_t x, int shift) { return (uint32_t(x) * 0x9E3779B1u) >> shift; }

// membership of members tails[r0, r1) (ascending ids) in `words` words
struct NaSet {
  int32_t *words;
  int32_t lo, hi;
  uint32_t mask;
  int shift;
  bool bitmap;
  __device__ __forceinline__ int layout(const int64_t *__restrict__ tails, int64_t r0, int64_t r1, int nwords) {
    lo = int32_t(tails[r0]);
    hi = int32_t(tails[r1 - 1]);
    const int64_t range = int64_t(hi) - lo + 1;
    bitmap = range <= int64_t(nwords) * 32;
    if (bitmap) return int((range + 31) >> 5);
    int lg = 6;
    while ((int64_t(1) << lg) < 4 * (r1 - r0)) lg++;
    mask = (1u << lg) - 1;
    shift = 32 - lg;
    return 1 << lg;
  }
  __device__ __forceinline__ void insert(int32_t x) const {
    if (bitmap) {
      const uint32_t d = uint32_t(x - lo);
      if (d > uint32_t(hi - lo)) return;  // only on a row out of order (rejected by k_na_check)
      atomicOr(reinterpret_cast<unsigned int *>(&words[d >> 5]), 1u << (d & 31));
      return;
    }
    uint32_t h = na_hash(x, shift);
    while (true) {
      const int32_t old = atomicCAS(&words[h], kEmpty, x);
      if (old == kEmpty || old == x) return;
      h = (h + 1) & mask;
    }
  }
  __device__ __forceinline__ int contains(int32_t x) const {
    const uint32_t d = uint32_t(x - lo);
    if (d > uint32_t(hi - lo)) return 0;
    if (bitmap) return (words[d >> 5] >> (d & 31)) & 1;
    uint32_t h = na_hash(x, shift);
    while (true) {
      const int32_t k = words[h];
      if (k == x) return 1;
      if (k == kEmpty) return 0;
      h = (h + 1) & mask;
    }
  }
};

// The suffix of row u after its neighbour v (v > u): [position of v + 1, end).
// A row without v means the input is not symmetric: flag it, count nothing.
__device__ __forceinline__ void suffix_after(const int64_t *__restrict__ off, const int64_t *__restrict__ tails,
                                             const Scratch &sc, int64_t u, int64_t v, int64_t &s, int64_t &e) {
  int64_t lo = off[u] + sc.split[u], hi = off[u + 1];
  e = hi;
  while (lo < hi) {
    const int64_t mid = lo + (hi - lo) / 2;
    if (tails[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  if (lo >= e || tails[lo] != v) {
    atomicOr(&sc.hdr->err, 1);
    s = e;
    return;
  }
  s = lo + 1;
}

// One warp: the in-neighbours u = tails[k], k in [k0, k1) step kstep (32-wide
// batches), each streaming the suffix of its row after v through the set.
__device__ __forceinline__ int64_t na_stream(const int64_t *__restrict__ off, const int64_t *__restrict__ tails,
                                             const Scratch &sc, int64_t v, int64_t k0, int64_t k1, int64_t kstep,
                                             const NaSet &m, int lane) {
  int64_t hits = 0;
  for (int64_t kb = k0; kb < k1; kb += kstep) {
    int64_t s = 0, e = 0;
    const int64_t k = kb + lane;
    if (k < k1) suffix_after(off, tails, sc, tails[k], v, s, e);
    const int nb = (k1 - kb < 32) ? int(k1 - kb) : 32;
    for (int j = 0; j < nb; j++) {
      const int64_t sj = __shfl_sync(0xffffffffu, s, j), ej = __shfl_sync(0xffffffffu, e, j);
      for (int64_t p = sj + lane; p < ej; p += 32) hits += m.contains(int32_t(tails[p]));
    }
  }
  return hits;
}

// warp pass: every head with 1..kWarpD out-neighbours and an in-neighbour
__global__ void __launch_bounds__(kThreads) k_na_warp(int64_t nv, const int64_t *__restrict__ off,
                                                      const int64_t *__restrict__ tails, Scratch sc) {
  __shared__ int32_t words_all[kWarps * kWarpWords];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int32_t *words = words_all + warp * kWarpWords;
  int64_t hits = 0;
  if (sc.hdr->err) return;  // the input check failed
  while (true) {
    unsigned long long b = 0;
    if (lane == 0) b = atomicAdd(&sc.hdr->cursor_w, (unsigned long long)kHeadBatch);
    const int64_t v0 = int64_t(__shfl_sync(0xffffffffu, b, 0));
    if (v0 >= nv) break;
    const int64_t v1 = (v0 + kHeadBatch < nv) ? v0 + kHeadBatch : nv;
    for (int64_t v = v0; v < v1; v++) {
      const int64_t e0 = off[v], mid = e0 + sc.split[v], e1 = off[v + 1];
      if (mid == e0 || e1 == mid || e1 - mid > kWarpD) continue;  // no in-neighbour, no out-list, or heavy
      NaSet m;
      m.words = words;
      const int nclear = m.layout(tails, mid, e1, kWarpWords);
      __syncwarp();
      for (int i = lane; i < nclear; i += 32) words[i] = m.bitmap ? 0 : kEmpty;
      __syncwarp();
      for (int64_t p = mid + lane; p < e1; p += 32) m.insert(int32_t(tails[p]));
      __syncwarp();
      hits += na_stream(off, tails, sc, v, e0, mid, 32, m, lane);
    }
  }
  for (int o = 16; o; o >>= 1) hits += __shfl_xor_sync(0xffffffffu, hits, o);
  if (lane == 0 && hits) atomicAdd(&sc.hdr->triangles, (unsigned long long)hits);
}

// CTA pass: the heavy heads, N+(v) in parts of kBlockPart members
__global__ void __launch_bounds__(kThreads) k_na_cta(const int64_t *__restrict__ off,
                                                     const int64_t *__restrict__ tails, Scratch sc) {
  __shared__ int32_t words[kBlockWords];
  __shared__ int64_t s_head;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t n_heavy = sc.hdr->err ? 0 : int64_t(sc.hdr->n_heavy);  // nothing when the input check failed
  int64_t hits = 0;
  while (true) {
    if (tid == 0) s_head = int64_t(atomicAdd(&sc.hdr->cursor_c, 1ull));
    __syncthreads();
    const int64_t h = s_head;
    __syncthreads();  // everyone read s_head before thread 0 may overwrite it
    if (h >= n_heavy) break;
    const int64_t v = sc.heavy[h];
    const int64_t e0 = off[v], mid = e0 + sc.split[v], e1 = off[v + 1];
    for (int64_t r0 = mid; r0 < e1; r0 += kBlockPart) {
      const int64_t r1 = (r0 + kBlockPart < e1) ? r0 + kBlockPart : e1;
      NaSet m;
      m.words = words;
      const int nclear = m.layout(tails, r0, r1, kBlockWords);
      for (int i = tid; i < nclear; i += kThreads) words[i] = m.bitmap ? 0 : kEmpty;
      __syncthreads();
      for (int64_t p = r0 + tid; p < r1; p += kThreads) m.insert(int32_t(tails[p]));
      __syncthreads();
      hits += na_stream(off, tails, sc, v, e0 + 32 * warp, mid, 32 * kWarps, m, lane);
      __syncthreads();
    }
  }
  for (int o = 16; o; o >>= 1) hits += __shfl_xor_sync(0xffffffffu, hits, o);
  if (lane == 0 && hits) atomicAdd(&sc.hdr->triangles, (unsigned long long)hits);
}

// the result, only when every check passed: on an error *out keeps its value
__global__ void k_na_finish(const Header *hdr, int64_t *out, int accumulate) {
  if (hdr->err) return;
  const int64_t t = int64_t(hdr->triangles);
  *out = accumulate ? *out + t : t;
}

// Address of g_scratch on each device, looked up once per device (with that
// device current) the first time the entry point runs there.
std::mutex g_mu;
unsigned char *g_base[64] = {nullptr};

static cudaError_t scratch_base(int dev, unsigned char **out) {
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_base[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) return e;
    g_base[dev] = static_cast<unsigned char *>(p);
  }
  *out = g_base[dev];
  return cudaSuccess;
}

}  // namespace nalloc
}  // namespace xt

extern "C" xt_status xt_count_device_static(int64_t nv, const int64_t *d_indices, const int64_t *d_edge_list,
                                            int64_t *d_count, int accumulate, void *cuda_stream) {
  using namespace xt::nalloc;
  if (nv < 1 || !d_indices || !d_edge_list || !d_count) return XT_ERR_INVALID;
  if (nv > kMaxNv) return XT_ERR_OVERFLOW;  // the fixed scratch holds 8 bytes per vertex
  // an error left pending by the caller's own earlier work is not this call's:
  // report it without clearing it, before launching anything
  if (cudaPeekAtLastError() != cudaSuccess) return XT_ERR_CUDA;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return XT_ERR_NO_DEVICE;
  unsigned char *base = nullptr;
  if (scratch_base(dev, &base) != cudaSuccess) {
    cudaGetLastError();
    return XT_ERR_CUDA;
  }
  cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
  const Scratch sc = carve(base, nv);
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) {
    cudaGetLastError();
    return XT_ERR_CUDA;
  }
  k_na_init<<<1, 1, 0, st>>>(sc.hdr);
  const int64_t gw = (nv * 32 + kThreads - 1) / kThreads;
  const unsigned grid_rows = unsigned(gw < int64_t(sms) * 32 ? gw : int64_t(sms) * 32);
  k_na_check<<<grid_rows, kThreads, 0, st>>>(nv, d_indices, d_edge_list, sc.hdr);
  k_na_back<<<grid_rows, kThreads, 0, st>>>(nv, d_indices, d_edge_list, sc.hdr);
  const int64_t gs = (nv + kThreads - 1) / kThreads;
  k_na_split<<<unsigned(gs < int64_t(sms) * 32 ? gs : int64_t(sms) * 32), kThreads, 0, st>>>(nv, d_indices,
                                                                                             d_edge_list, sc);
  k_na_warp<<<unsigned(sms * 8), kThreads, 0, st>>>(nv, d_indices, d_edge_list, sc);
  k_na_cta<<<unsigned(sms * 4), kThreads, 0, st>>>(d_indices, d_edge_list, sc);
  k_na_finish<<<1, 1, 0, st>>>(sc.hdr, d_count, accumulate);
  if (cudaGetLastError() != cudaSuccess) return XT_ERR_CUDA;  // nothing was pending at entry: these launches
  int err = 0;
  if (cudaMemcpyAsync(&err, &sc.hdr->err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    cudaGetLastError();
    return XT_ERR_CUDA;
  }
  return err ? XT_ERR_INVALID : XT_OK;
}
