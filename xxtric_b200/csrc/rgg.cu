// The reference's random geometric graph generated on the device.
//
// Replaces the host loops of GenerateRGG::generate (graph.hpp:745-1364) and
// its LCG (utils.hpp:245-430) for the -n path with -p 0, as nprocs strip ranks
// would build the graph under mpiexec -n nprocs. The edge set is bit-for-bit
// the reference's (and the host restatement's, xt_rgg_generate):
//
//   * coordinates: rank r's LCG stream x_{i+1} = 16807 x_i % (2^31 - 1)
//     starts at x0[r] (the host set-up, xt_rgg_setup, computes it exactly as
//     the reference's overflowing 2x2 prefix does, sign included). The
//     magnitude of element i is |x0[r]| * 16807^i mod (2^31 - 1), computed
//     per element from a table of 16807^(2^k) (the reference's recurrence
//     never overflows 64 bits, and C's % keeps the sign of a negative stream,
//     so the magnitudes are the same integers). X = the first n of the rank's 2n doubles
//     |x| / (2^31 - 1), Y = the rest rescaled into the rank's strip;
//   * an edge for every pair whose sqrt(dx*dx + dy*dy) <= r, cross-strip
//     pairs only between adjacent strips and only when the local indices
//     differ (graph.hpp:919-948, 976-1036).
//
// The double arithmetic uses the explicitly rounded intrinsics (__dmul_rn,
// __dadd_rn, __dsub_rn, __dsqrt_rn), so no product is fused into an FMA and
// every operation rounds as the host's IEEE arithmetic does. Pairs are found
// through a grid of cells no smaller than r (points sorted by cell), one
// thread per point, in two passes: count, then write at the scanned offsets.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include "xt_internal.cuh"

namespace xt {

constexpr uint64_t kLcgM = 2147483647ULL;  // 2^31 - 1
constexpr uint64_t kLcgA = 16807ULL;

struct LcgPow {
  uint64_t p[40];  // 16807^(2^k) mod (2^31 - 1)
};

__device__ __forceinline__ uint64_t lcg_mulmod(uint64_t a, uint64_t b) { return (a * b) % kLcgM; }

// coordinates of point r * n + i from element j of rank r's stream: X for j < n,
// Y (rescaled into the strip) for j >= n
__global__ void k_rgg_coords(int64_t n, int P, const int64_t *__restrict__ x0, const double *__restrict__ lo,
                             double range, double mult, const LcgPow pw, double *__restrict__ X,
                             double *__restrict__ Y) {
  const int64_t total = int64_t(P) * 2 * n;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = t / (2 * n), j = t % (2 * n);
    // a rank's first value may be negative (the reference's % of a wrapped
    // int64); its stream then stays negative, -(|x| 16807^j mod m), and the
    // coordinate takes the magnitude
    uint64_t x = uint64_t(x0[r] < 0 ? -x0[r] : x0[r]);
    for (int k = 0; (int64_t(1) << k) <= j; k++)
      if ((j >> k) & 1) x = lcg_mulmod(x, pw.p[k]);
    const double d = __dmul_rn(double(x), mult);  // |x| / (1 + (2^31 - 2)); x >= 0
    if (j < n) X[r * n + j] = d;
    else Y[r * n + (j - n)] = __dadd_rn(lo[r], __dmul_rn(range, d));
  }
}

__device__ __forceinline__ int32_t rgg_cell1(double v, int gc) {
  int64_t c = int64_t(__dmul_rn(v, double(gc)));  // truncation, as the host's cast
  return int32_t(c < 0 ? 0 : (c >= gc ? gc - 1 : c));
}

__global__ void k_rgg_cells(int64_t nv, int gc, const double *__restrict__ X, const double *__restrict__ Y,
                            uint32_t *__restrict__ cell, int32_t *__restrict__ ids,
                            unsigned long long *__restrict__ ccount) {
  for (int64_t a = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; a < nv; a += int64_t(gridDim.x) * blockDim.x) {
    const uint32_t c = uint32_t(rgg_cell1(Y[a], gc)) * uint32_t(gc) + uint32_t(rgg_cell1(X[a], gc));
    cell[a] = c;
    ids[a] = int32_t(a);
    atomicAdd(&ccount[c], 1ull);
  }
}

// Pass 1 (src == null): the pairs (a, b), b > a, of every point a into cnt[a].
// Pass 2: writes them at out_off[a].
__global__ void k_rgg_pairs(int64_t nv, int64_t n, int gc, double rn, const double *__restrict__ X,
                            const double *__restrict__ Y, const uint32_t *__restrict__ cell,
                            const int32_t *__restrict__ order, const unsigned long long *__restrict__ cstart,
                            int64_t *__restrict__ cnt, const int64_t *__restrict__ out_off,
                            int32_t *__restrict__ src, int32_t *__restrict__ dst) {
  for (int64_t a = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; a < nv; a += int64_t(gridDim.x) * blockDim.x) {
    const int64_t ra = a / n, ia = a % n;
    const int32_t c = int32_t(cell[a]), cx = c % gc, cy = c / gc;
    const double xa = X[a], ya = Y[a];
    int64_t k = 0, o = src ? out_off[a] : 0;
    for (int dy = -1; dy <= 1; dy++) {
      const int32_t ny = cy + dy;
      if (ny < 0 || ny >= gc) continue;
      for (int dx = -1; dx <= 1; dx++) {
        const int32_t nx = cx + dx;
        if (nx < 0 || nx >= gc) continue;
        const int64_t c2 = int64_t(ny) * gc + nx;
        for (unsigned long long q = cstart[c2]; q < cstart[c2 + 1]; q++) {
          const int64_t b = order[q];
          if (b <= a) continue;
          const int64_t rb = b / n, ib = b % n;
          if (rb != ra) {
            if (rb - ra != 1 && ra - rb != 1) continue;  // only adjacent strips exchange ghosts
            if (ia == ib) continue;                      // j > i on both sides drops equal indices
          }
          const double ddx = __dsub_rn(xa, X[b]), ddy = __dsub_rn(ya, Y[b]);
          const double ed = __dsqrt_rn(__dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy)));
          if (ed <= rn) {
            if (src) {
              src[o + k] = int32_t(a);
              dst[o + k] = int32_t(b);
            }
            k++;
          }
        }
      }
    }
    if (!src) cnt[a] = k;
  }
}

static unsigned rgg_grid(const Ctx *c, int64_t n) {
  int64_t g = (n + 255) / 256, cap = int64_t(c->sm_count) * 16;
  return unsigned(g < 1 ? 1 : (g > cap ? cap : g));
}

xt_status gen_rgg(Ctx *c, int64_t nv, int nprocs, double radius, int64_t cap, int64_t *n_pairs, int32_t *d_src,
                  int32_t *d_dst) {
  if (!n_pairs || nv < 1 || nv > (int64_t(1) << 31) - 1 || nprocs < 1)
    return set_error(c, XT_ERR_INVALID, "xt_gen_rgg: bad arguments");
  std::vector<int64_t> x0(static_cast<size_t>(nprocs));
  std::vector<double> lo(static_cast<size_t>(nprocs));
  double rn = 0, range = 0;
  if (xt_rgg_setup(nv, nprocs, radius, &rn, x0.data(), lo.data(), &range) != XT_OK)
    return set_error(c, XT_ERR_INVALID, "xt_gen_rgg: nprocs must be a power of two dividing nv, and r < 1/nprocs");
  const int64_t n = nv / nprocs;
  LcgPow pw;
  pw.p[0] = kLcgA;
  for (int k = 1; k < 40; k++) pw.p[k] = (pw.p[k - 1] * pw.p[k - 1]) % kLcgM;
  const double mult = 1.0 / double(1.0 + double(int64_t(kLcgM) - 1));
  // a grid of cells no smaller than r (the host generator's choice)
  int64_t gc = int64_t(std::floor(1.0 / (rn * 1.0001)));
  gc = std::max<int64_t>(1, std::min<int64_t>(gc, 8192));
  const int64_t ncell = gc * gc;
  double *X = nullptr, *Y = nullptr, *d_lo = nullptr;
  int64_t *d_x0 = nullptr, *cnt = nullptr, *off = nullptr;
  uint32_t *cell = nullptr, *cell2 = nullptr;
  int32_t *ids = nullptr, *order = nullptr;
  unsigned long long *ccount = nullptr, *cstart = nullptr;
  void *tmp = nullptr;
  xt_status s = XT_OK;
  do {
    if ((s = dalloc_n(c, &X, size_t(nv))) != XT_OK) break;
    if ((s = dalloc_n(c, &Y, size_t(nv))) != XT_OK) break;
    if ((s = dalloc_n(c, &d_x0, size_t(nprocs))) != XT_OK) break;
    if ((s = dalloc_n(c, &d_lo, size_t(nprocs))) != XT_OK) break;
    if ((s = dalloc_n(c, &cell, size_t(nv))) != XT_OK) break;
    if ((s = dalloc_n(c, &cell2, size_t(nv))) != XT_OK) break;
    if ((s = dalloc_n(c, &ids, size_t(nv))) != XT_OK) break;
    if ((s = dalloc_n(c, &order, size_t(nv))) != XT_OK) break;
    if ((s = dalloc_n(c, &ccount, size_t(ncell + 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &cstart, size_t(ncell + 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &cnt, size_t(nv + 1))) != XT_OK) break;
    if ((s = dalloc_n(c, &off, size_t(nv + 1))) != XT_OK) break;
    cudaError_t e = cudaMemcpyAsync(d_x0, x0.data(), sizeof(int64_t) * nprocs, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_lo, lo.data(), sizeof(double) * nprocs, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(ccount, 0, sizeof(unsigned long long) * (ncell + 1), c->stream);
    if ((s = cuda_status(c, e, "rgg set-up")) != XT_OK) break;
    k_rgg_coords<<<counted(c, rgg_grid(c, 2 * nv)), 256, 0, c->stream>>>(n, nprocs, d_x0, d_lo, range, mult, pw, X,
                                                                          Y);
    k_rgg_cells<<<counted(c, rgg_grid(c, nv)), 256, 0, c->stream>>>(nv, int(gc), X, Y, cell, ids, ccount);
    if ((s = cuda_status(c, cudaGetLastError(), "rgg cells")) != XT_OK) break;
    // points ordered by cell (stable: ids ascend within a cell), cell starts
    size_t bytes = 0, b2 = 0;
    int end_bit = 1;
    while (end_bit < 32 && (int64_t(1) << end_bit) < ncell) end_bit++;
    e = cub::DeviceRadixSort::SortPairs(nullptr, bytes, cell, cell2, ids, order, nv, 0, end_bit, c->stream);
    if (e == cudaSuccess)
      e = cub::DeviceScan::ExclusiveSum(nullptr, b2, ccount, cstart, ncell + 1, c->stream);
    if ((s = cuda_status(c, e, "rgg sort")) != XT_OK) break;
    if ((s = dalloc(c, &tmp, std::max(bytes, b2))) != XT_OK) break;
    e = cub::DeviceRadixSort::SortPairs(tmp, bytes, cell, cell2, ids, order, nv, 0, end_bit, c->stream);
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp, b2, ccount, cstart, ncell + 1, c->stream);
    if ((s = cuda_status(c, e, "rgg sort")) != XT_OK) break;
    // pass 1: pairs per point, scanned into output offsets
    k_rgg_pairs<<<counted(c, rgg_grid(c, nv)), 256, 0, c->stream>>>(nv, n, int(gc), rn, X, Y, cell, order, cstart,
                                                                     cnt, nullptr, nullptr, nullptr);
    if ((s = cuda_status(c, cudaMemsetAsync(cnt + nv, 0, sizeof(int64_t), c->stream), "memset")) != XT_OK) break;
    dfree(c, tmp);
    tmp = nullptr;
    size_t b3 = 0;
    if ((s = cuda_status(c, cub::DeviceScan::ExclusiveSum(nullptr, b3, cnt, off, nv + 1, c->stream), "scan")) !=
        XT_OK)
      break;
    if ((s = dalloc(c, &tmp, b3)) != XT_OK) break;
    if ((s = cuda_status(c, cub::DeviceScan::ExclusiveSum(tmp, b3, cnt, off, nv + 1, c->stream), "scan")) != XT_OK)
      break;
    int64_t total = 0;
    if ((s = cuda_status(c, cudaMemcpyAsync(&total, off + nv, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream),
                         "D2H")) != XT_OK)
      break;
    if ((s = cuda_status(c, cudaStreamSynchronize(c->stream), "sync")) != XT_OK) break;
    *n_pairs = total;
    if (!d_src) break;  // sizing call
    if (!d_dst || cap < total) {
      s = set_error(c, XT_ERR_OVERFLOW, "xt_gen_rgg: the output holds fewer rows than the graph has pairs");
      break;
    }
    k_rgg_pairs<<<counted(c, rgg_grid(c, nv)), 256, 0, c->stream>>>(nv, n, int(gc), rn, X, Y, cell, order, cstart,
                                                                     nullptr, off, d_src, d_dst);
    s = cuda_status(c, cudaGetLastError(), "rgg pairs");
  } while (0);
  dfree(c, tmp);
  dfree(c, X);
  dfree(c, Y);
  dfree(c, d_x0);
  dfree(c, d_lo);
  dfree(c, cell);
  dfree(c, cell2);
  dfree(c, ids);
  dfree(c, order);
  dfree(c, ccount);
  dfree(c, cstart);
  dfree(c, cnt);
  dfree(c, off);
  return s;
}

}  // namespace xt
