// Deterministic synthetic-graph generators on the device: R-MAT, Chung-Lu
// and Erdos-Renyi graphs. The reference
// generates only its random geometric graph (graph.hpp:745-1364, restated
// on the host in host/host_io.cpp) and otherwise reads edge lists from
// files (cugraph/cug_triangle_count.py:23-25). Every edge is a
// pure function of (seed, edge index), so the same seed yields the same
// edge list on any GPU and in the CPU oracle's twins of these functions.
// Integer arithmetic only (quadrant choice by 64x64->128 high products,
// endpoint draws from an integer CDF), so no rounding mode can differ.
#include "xt_internal.cuh"
#include "xt_rng.cuh"

namespace xt {

constexpr uint64_t kStreamRmat = 1, kStreamCL = 2, kStreamER = 3;
constexpr uint64_t kPermSalt = 0x5bd1e9955bd1e995ULL;

__global__ void k_gen_rmat(int scale, int64_t ne, uint64_t seed, uint64_t pa, uint64_t pb, uint64_t pc, uint64_t pd,
                           uint64_t base, uint64_t span, int permute, int32_t *__restrict__ src,
                           int32_t *__restrict__ dst) {
  const uint64_t p[4] = {pa, pb, pc, pd};
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < ne; e += int64_t(gridDim.x) * blockDim.x) {
    uint64_t u = 0, v = 0;
    for (int l = 0; l < scale; l++) {
      const uint64_t rn = crand(seed, kStreamRmat, uint64_t(e) * 128u + 2u * uint64_t(l));
      const uint64_t rq = crand(seed, kStreamRmat, uint64_t(e) * 128u + 2u * uint64_t(l) + 1u);
      uint64_t w[4], s = 0;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const uint64_t nz = (rn >> (8 * q)) & 0xffu;
        w[q] = p[q] * (base + (nz * span) / 255u);
        s += w[q];
      }
      const uint64_t x = __umul64hi(rq, s);
      const int quad = (x < w[0]) ? 0 : (x < w[0] + w[1]) ? 1 : (x < w[0] + w[1] + w[2]) ? 2 : 3;
      u |= uint64_t(quad >> 1) << l;
      v |= uint64_t(quad & 1) << l;
    }
    if (permute) {
      u = perm_bits(u, scale, seed ^ kPermSalt);
      v = perm_bits(v, scale, seed ^ kPermSalt);
    }
    src[e] = int32_t(u);
    dst[e] = int32_t(v);
  }
}

__device__ __forceinline__ int64_t cdf_find(const uint64_t *__restrict__ cdf, int64_t n, uint64_t x) {
  int64_t lo = 0, hi = n;
  while (hi - lo > 1) {
    int64_t mid = lo + (hi - lo) / 2;
    if (cdf[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

__global__ void k_gen_chunglu(int64_t n, const uint64_t *__restrict__ cdf, int64_t ne, uint64_t seed, int permute,
                              int bits, int32_t *__restrict__ src, int32_t *__restrict__ dst) {
  const uint64_t total = cdf[n];
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < ne; e += int64_t(gridDim.x) * blockDim.x) {
    uint64_t a = uint64_t(cdf_find(cdf, n, __umul64hi(crand(seed, kStreamCL, 2u * uint64_t(e)), total)));
    uint64_t b = uint64_t(cdf_find(cdf, n, __umul64hi(crand(seed, kStreamCL, 2u * uint64_t(e) + 1u), total)));
    if (permute) {
      a = perm_bits(a, bits, seed ^ kPermSalt);
      b = perm_bits(b, bits, seed ^ kPermSalt);
    }
    src[e] = int32_t(a);
    dst[e] = int32_t(b);
  }
}

__global__ void k_gen_er(int64_t n, int64_t ne, uint64_t seed, int32_t *__restrict__ src,
                         int32_t *__restrict__ dst) {
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < ne; e += int64_t(gridDim.x) * blockDim.x) {
    src[e] = int32_t(__umul64hi(crand(seed, kStreamER, 2u * uint64_t(e)), uint64_t(n)));
    dst[e] = int32_t(__umul64hi(crand(seed, kStreamER, 2u * uint64_t(e) + 1u), uint64_t(n)));
  }
}

static unsigned gen_grid(const Ctx *c, int64_t n) {
  int64_t g = (n + 255) / 256, cap = int64_t(c->sm_count) * 16;
  return unsigned(g < 1 ? 1 : (g > cap ? cap : g));
}

xt_status gen_rmat(Ctx *c, int scale, int64_t ne, uint64_t seed, int a16, int b16, int c16, int noise_pct,
                   int permute, int32_t *d_src, int32_t *d_dst) {
  if (scale < 1 || scale > 31 || ne < 0 || !d_src || !d_dst || a16 < 0 || b16 < 0 || c16 < 0 ||
      a16 + b16 + c16 > 65536 || noise_pct < 0 || noise_pct > 100)
    return set_error(c, XT_ERR_INVALID, "xt_gen_rmat: bad arguments");
  const uint64_t base = uint64_t(100 - noise_pct) * 256u, span = uint64_t(noise_pct) * 512u;
  if (ne)
    k_gen_rmat<<<counted(c, gen_grid(c, ne)), 256, 0, c->stream>>>(scale, ne, seed, uint64_t(a16), uint64_t(b16), uint64_t(c16),
                                                        uint64_t(65536 - a16 - b16 - c16), base, span, permute,
                                                        d_src, d_dst);
  XT_CUDA(c, cudaGetLastError());
  return XT_OK;
}

xt_status gen_chunglu(Ctx *c, int64_t n, const uint64_t *cdf, int64_t ne, uint64_t seed, int permute,
                      int32_t *d_src, int32_t *d_dst) {
  if (n < 1 || n > (int64_t(1) << 31) - 1 || ne < 0 || !cdf || !d_src || !d_dst)
    return set_error(c, XT_ERR_INVALID, "xt_gen_chunglu: bad arguments");
  int bits = 0;
  while ((int64_t(1) << bits) < n) bits++;
  if (permute && (int64_t(1) << bits) != n)
    return set_error(c, XT_ERR_INVALID, "xt_gen_chunglu: permute needs a power-of-two n");
  uint64_t *d_cdf = nullptr;
  XT_TRY(dalloc_n(c, &d_cdf, size_t(n + 1)));
  cudaError_t e = cudaMemcpyAsync(d_cdf, cdf, sizeof(uint64_t) * (n + 1), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess && ne) {
    k_gen_chunglu<<<counted(c, gen_grid(c, ne)), 256, 0, c->stream>>>(n, d_cdf, ne, seed, permute, bits, d_src, d_dst);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);  // host cdf may be freed after return
  dfree(c, d_cdf);
  XT_CUDA(c, e);
  return XT_OK;
}

xt_status gen_er(Ctx *c, int64_t n, int64_t ne, uint64_t seed, int32_t *d_src, int32_t *d_dst) {
  if (n < 1 || n > (int64_t(1) << 31) - 1 || ne < 0 || !d_src || !d_dst)
    return set_error(c, XT_ERR_INVALID, "xt_gen_er: bad arguments");
  if (ne) k_gen_er<<<counted(c, gen_grid(c, ne)), 256, 0, c->stream>>>(n, ne, seed, d_src, d_dst);
  XT_CUDA(c, cudaGetLastError());
  return XT_OK;
}

}  // namespace xt
