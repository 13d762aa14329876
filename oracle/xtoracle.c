/*
 * xtoracle.c — TEST INFRASTRUCTURE ONLY. CPU restatement of the reference's
 * counting path (sg0/xxtric xxtric.hpp) and of the deterministic generators
 * whose GPU twins live in the product. Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg load this library, and only as a checker.
 *
 * Pinned against the reference's own CPU binary (oracle/_ref/tric) on the
 * golden fixtures in tests/golden/ (K4, K5, isolated tail, Erdos-Renyi,
 * the reference's LCG random geometric graphs, amazon0302).
 */
#include "xtoracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* ======================================================================== */
/* counting                                                                  */
/* ======================================================================== */

/* check_edgelist (xxtric.hpp:516-545): first/last shortcut then a binary
 * search of w in the sorted row of v. Reads that the reference would make
 * outside the tails array (a degree-0 row) return 0 here. */
static int xo_check_edgelist(const int64_t *off, const int64_t *tails, int64_t ne, int64_t v, int64_t w) {
  int64_t beg = off[v], end = off[v + 1];
  int64_t first = (beg >= 0 && beg < ne) ? tails[beg] : 0;
  int64_t last = (end - 1 >= 0 && end - 1 < ne) ? tails[end - 1] : 0;
  if (w == last || w == first) return 1;
  if (w > first && w < last) {
    int64_t mid = beg + (end - beg) / 2;
    while (end > beg) {
      int64_t t = tails[mid];
      if (t == w) return 1;
      if (t < w) beg = mid + 1;
      else end = mid;
      mid = beg + (end - beg) / 2;
    }
  }
  return 0;
}

int64_t xo_count_xxtric(int64_t nv, const int64_t *off, const int64_t *tails) {
  if (nv <= 0) return 0;
  const int64_t ne = off[nv];
  /* erange_ (xxtric.hpp:60-75): min/max neighbour; rows of one entry skip */
  int64_t *erange = (int64_t *)calloc((size_t)(2 * nv), sizeof(int64_t));
  if (!erange) return -1;
  for (int64_t i = 0; i < nv; i++) {
    int64_t e0 = off[i], e1 = off[i + 1];
    if (e0 + 1 == e1) continue;
    erange[2 * i] = (e0 >= 0 && e0 < ne) ? tails[e0] : 0;
    erange[2 * i + 1] = (e1 - 1 >= 0 && e1 - 1 < ne) ? tails[e1 - 1] : 0;
  }
  int64_t count = 0;
  /* local count loop (xxtric.hpp:150-207) at one rank: every v is local */
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : count)
  for (int64_t i = 0; i < nv; i++) {
    int64_t e0 = off[i], e1 = off[i + 1];
    if (e0 + 1 == e1) continue;
    for (int64_t m = e0; m < e1 - 1; m++) {
      int64_t v = tails[m];
      if (i >= v) continue;
      for (int64_t n = m + 1; n < e1; n++) {
        int64_t w = tails[n];
        if (!(w <= erange[2 * v + 1])) break; /* edge_within_max */
        if (!(w >= erange[2 * v])) continue;  /* edge_above_min */
        if (xo_check_edgelist(off, tails, ne, v, w)) count += 1;
      }
    }
  }
  free(erange);
  return count;
}

/* first index in [lo,hi) of sorted a with a[k] > x */
static int64_t xo_upper(const int64_t *a, int64_t lo, int64_t hi, int64_t x) {
  while (lo < hi) {
    int64_t mid = lo + (hi - lo) / 2;
    if (a[mid] <= x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

int64_t xo_count_merge(int64_t nv, const int64_t *off, const int64_t *tails, int64_t *pv) {
  if (pv) memset(pv, 0, sizeof(int64_t) * (size_t)(nv > 0 ? nv : 0));
  int64_t total = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : total)
  for (int64_t u = 0; u < nv; u++) {
    const int64_t a0 = xo_upper(tails, off[u], off[u + 1], u), a1 = off[u + 1];
    for (int64_t p = a0; p < a1; p++) {
      const int64_t v = tails[p];
      int64_t i = p + 1, j = xo_upper(tails, off[v], off[v + 1], v);
      const int64_t je = off[v + 1];
      int64_t local = 0;
      while (i < a1 && j < je) {
        int64_t x = tails[i], y = tails[j];
        if (x < y) i++;
        else if (y < x) j++;
        else {
          local++;
          if (pv) {
#pragma omp atomic
            pv[x] += 1;
          }
          i++; j++;
        }
      }
      if (pv && local) {
#pragma omp atomic
        pv[v] += local;
#pragma omp atomic
        pv[u] += local;
      }
      total += local;
    }
  }
  return total;
}

/* Triangles through each selected vertex s: edges among N(s), found by
 * marking N(s) in a bitmap and counting marked entries of every N(x), x in
 * N(s) (each such edge is seen from both ends). Cost: sum of d(x) over
 * x in N(s), so hubs of Chung-Lu graphs stay cheap. */
void xo_local_counts(int64_t nv, const int64_t *off, const int64_t *tails, int64_t nsel, const int64_t *sel,
                     int64_t *out) {
#pragma omp parallel
  {
    uint64_t *mark = (uint64_t *)calloc((size_t)(nv / 64 + 1), sizeof(uint64_t));
#pragma omp for schedule(dynamic, 1)
    for (int64_t k = 0; k < nsel; k++) {
      const int64_t s = sel[k];
      const int64_t a0 = off[s], a1 = off[s + 1];
      for (int64_t p = a0; p < a1; p++) mark[tails[p] >> 6] |= (uint64_t)1 << (tails[p] & 63);
      int64_t twice = 0;
      for (int64_t p = a0; p < a1; p++) {
        const int64_t v = tails[p];
        for (int64_t j = off[v]; j < off[v + 1]; j++) twice += (int64_t)((mark[tails[j] >> 6] >> (tails[j] & 63)) & 1);
      }
      for (int64_t p = a0; p < a1; p++) mark[tails[p] >> 6] = 0;
      out[k] = twice / 2;
    }
    free(mark);
  }
}

/* Triangles on every edge: for each CSR entry (a, b), |N(a) and N(b)|, by
 * marking N(a) and counting the marked entries of N(b). The per-edge form of
 * the per-vertex counts (a triangle credits each of its three edges). */
void xo_edge_support(int64_t nv, const int64_t *off, const int64_t *tails, int64_t *out) {
#pragma omp parallel
  {
    uint64_t *mark = (uint64_t *)calloc((size_t)(nv / 64 + 1), sizeof(uint64_t));
#pragma omp for schedule(dynamic, 64)
    for (int64_t a = 0; a < nv; a++) {
      for (int64_t p = off[a]; p < off[a + 1]; p++) mark[tails[p] >> 6] |= (uint64_t)1 << (tails[p] & 63);
      for (int64_t p = off[a]; p < off[a + 1]; p++) {
        const int64_t b = tails[p];
        int64_t c = 0;
        for (int64_t j = off[b]; j < off[b + 1]; j++) c += (int64_t)((mark[tails[j] >> 6] >> (tails[j] & 63)) & 1);
        out[p] = c;
      }
      for (int64_t p = off[a]; p < off[a + 1]; p++) mark[tails[p] >> 6] = 0;
    }
    free(mark);
  }
}

/* ======================================================================== */
/* canonical CSR                                                             */
/* ======================================================================== */

static void xo_radix_u64(uint64_t *a, uint64_t *tmp, int64_t n, int bits) {
  uint64_t *src = a, *dst = tmp;
  for (int shift = 0; shift < bits; shift += 16) {
    int64_t *cnt = (int64_t *)calloc(65537, sizeof(int64_t));
    for (int64_t i = 0; i < n; i++) cnt[((src[i] >> shift) & 0xffff) + 1]++;
    for (int d = 0; d < 65536; d++) cnt[d + 1] += cnt[d];
    for (int64_t i = 0; i < n; i++) dst[cnt[(src[i] >> shift) & 0xffff]++] = src[i];
    free(cnt);
    uint64_t *t = src; src = dst; dst = t;
  }
  if (src != a) memcpy(a, src, sizeof(uint64_t) * (size_t)n);
}

int64_t xo_canon_csr(int64_t nv, int64_t ne, const int64_t *src, const int64_t *dst, int64_t *off,
                     int64_t *tails) {
  if (nv < 0 || nv > (int64_t)1 << 32) return -1;
  uint64_t *key = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(ne > 0 ? ne : 1));
  uint64_t *tmp = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(ne > 0 ? ne : 1));
  int64_t k = 0;
  for (int64_t e = 0; e < ne; e++) {
    int64_t a = src[e], b = dst[e];
    if (a < 0 || b < 0 || a >= nv || b >= nv) { free(key); free(tmp); return -1; }
    if (a == b) continue;
    uint64_t lo = (uint64_t)(a < b ? a : b), hi = (uint64_t)(a < b ? b : a);
    key[k++] = (lo << 32) | hi;
  }
  xo_radix_u64(key, tmp, k, 64);
  int64_t u = 0;
  for (int64_t i = 0; i < k; i++)
    if (i == 0 || key[i] != key[i - 1]) key[u++] = key[i];
  memset(off, 0, sizeof(int64_t) * (size_t)(nv + 1));
  for (int64_t i = 0; i < u; i++) {
    off[(key[i] >> 32) + 1]++;
    off[(key[i] & 0xffffffffu) + 1]++;
  }
  for (int64_t i = 0; i < nv; i++) off[i + 1] += off[i];
  int64_t *cur = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nv > 0 ? nv : 1));
  memcpy(cur, off, sizeof(int64_t) * (size_t)nv);
  for (int64_t i = 0; i < u; i++) {
    int64_t a = (int64_t)(key[i] >> 32), b = (int64_t)(key[i] & 0xffffffffu);
    tails[cur[a]++] = b;
    tails[cur[b]++] = a;
  }
  free(cur); free(key); free(tmp);
  return 2 * u;
}

/* ======================================================================== */
/* deterministic RNG                                                         */
/* ======================================================================== */

uint64_t xo_mix64(uint64_t z) {
  /* splitmix64 output function (Steele, Lea, Flood 2014; Vigna's constants) */
  z ^= z >> 30; z *= 0xbf58476d1ce4e5b9ULL;
  z ^= z >> 27; z *= 0x94d049bb133111ebULL;
  z ^= z >> 31;
  return z;
}

uint64_t xo_rand(uint64_t seed, uint64_t stream, uint64_t ctr) {
  uint64_t k = xo_mix64(seed * 0x9e3779b97f4a7c15ULL + stream + 0x632be59bd9b4e019ULL);
  return xo_mix64(k ^ (ctr * 0x9e3779b97f4a7c15ULL + 0xd1b54a32d192ed03ULL));
}

uint64_t xo_perm(uint64_t x, int bits, uint64_t seed) {
  const uint64_t mask = bits >= 64 ? ~0ULL : ((1ULL << bits) - 1);
  const int sh = (bits + 1) / 2;
  x &= mask;
  for (int r = 0; r < 4; r++) {
    uint64_t k = xo_mix64(seed + 0x9e3779b97f4a7c15ULL * (uint64_t)(r + 1));
    x = (x * (k | 1ULL)) & mask;
    x ^= (k >> 17) & mask;
    x ^= x >> sh;
  }
  return x & mask;
}

static inline uint64_t xo_mulhi(uint64_t a, uint64_t b) {
  return (uint64_t)(((unsigned __int128)a * (unsigned __int128)b) >> 64);
}

/* ======================================================================== */
/* generators                                                                */
/* ======================================================================== */

#define XO_STREAM_RMAT 1
#define XO_STREAM_CL 2
#define XO_STREAM_ER 3
#define XO_STREAM_RGG 4
#define XO_PERM_SALT 0x5bd1e9955bd1e995ULL

void xo_rmat_edges(int scale, uint64_t seed, int a16, int b16, int c16, int noise_pct, int permute, int64_t e0,
                   int64_t e1, int64_t *src, int64_t *dst) {
  const uint64_t p[4] = {(uint64_t)a16, (uint64_t)b16, (uint64_t)c16, (uint64_t)(65536 - a16 - b16 - c16)};
  const uint64_t base = (uint64_t)(100 - noise_pct) * 256u, span = (uint64_t)noise_pct * 512u;
#pragma omp parallel for schedule(static)
  for (int64_t e = e0; e < e1; e++) {
    uint64_t u = 0, v = 0;
    for (int l = 0; l < scale; l++) {
      uint64_t rn = xo_rand(seed, XO_STREAM_RMAT, (uint64_t)e * 128u + 2u * (uint64_t)l);
      uint64_t rq = xo_rand(seed, XO_STREAM_RMAT, (uint64_t)e * 128u + 2u * (uint64_t)l + 1u);
      uint64_t w[4], s = 0;
      for (int q = 0; q < 4; q++) {
        uint64_t nz = (rn >> (8 * q)) & 0xffu;
        w[q] = p[q] * (base + (nz * span) / 255u);
        s += w[q];
      }
      uint64_t x = xo_mulhi(rq, s);
      int quad = (x < w[0]) ? 0 : (x < w[0] + w[1]) ? 1 : (x < w[0] + w[1] + w[2]) ? 2 : 3;
      u |= (uint64_t)(quad >> 1) << l;
      v |= (uint64_t)(quad & 1) << l;
    }
    if (permute) {
      u = xo_perm(u, scale, seed ^ XO_PERM_SALT);
      v = xo_perm(v, scale, seed ^ XO_PERM_SALT);
    }
    src[e - e0] = (int64_t)u;
    dst[e - e0] = (int64_t)v;
  }
}

int64_t xo_chunglu_cdf(int64_t n, double gamma, double mean_deg, double max_deg, uint64_t *cdf) {
  /* expected degree w_i = max_deg * (1 + i/i0)^(-1/(gamma-1)); i0 by
   * bisection so that the integral approximation of the mean of w,
   * (max_deg/n) * int_0^n (1 + x/i0)^(-alpha) dx, equals mean_deg */
  const double alpha = 1.0 / (gamma - 1.0);
  double lo = 1e-9, hi = (double)n;
  for (int it = 0; it < 200; it++) {
    double i0 = 0.5 * (lo + hi), integral;
    if (fabs(1.0 - alpha) < 1e-12) integral = i0 * log(1.0 + (double)n / i0);
    else integral = i0 / (1.0 - alpha) * (pow(1.0 + (double)n / i0, 1.0 - alpha) - 1.0);
    if (max_deg * integral / (double)n > mean_deg) hi = i0;
    else lo = i0;
  }
  const double i0 = 0.5 * (lo + hi);
  cdf[0] = 0;
  for (int64_t i = 0; i < n; i++) {
    double w = max_deg * pow(1.0 + (double)i / i0, -alpha);
    uint64_t W = (uint64_t)llround(w * 1024.0);
    if (W < 1) W = 1;
    cdf[i + 1] = cdf[i] + W;
  }
  return (int64_t)llround((double)n * mean_deg / 2.0);
}

static inline int64_t xo_cdf_find(const uint64_t *cdf, int64_t n, uint64_t x) {
  int64_t lo = 0, hi = n; /* largest i with cdf[i] <= x, i in [0,n) */
  while (hi - lo > 1) {
    int64_t mid = lo + (hi - lo) / 2;
    if (cdf[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

void xo_chunglu_edges(int64_t n, const uint64_t *cdf, uint64_t seed, int permute, int64_t e0, int64_t e1,
                      int64_t *src, int64_t *dst) {
  const uint64_t total = cdf[n];
  int bits = 0;
  while (((int64_t)1 << bits) < n) bits++;
#pragma omp parallel for schedule(static)
  for (int64_t e = e0; e < e1; e++) {
    uint64_t a = (uint64_t)xo_cdf_find(cdf, n, xo_mulhi(xo_rand(seed, XO_STREAM_CL, 2u * (uint64_t)e), total));
    uint64_t b = (uint64_t)xo_cdf_find(cdf, n, xo_mulhi(xo_rand(seed, XO_STREAM_CL, 2u * (uint64_t)e + 1u), total));
    if (permute) {
      a = xo_perm(a, bits, seed ^ XO_PERM_SALT);
      b = xo_perm(b, bits, seed ^ XO_PERM_SALT);
    }
    src[e - e0] = (int64_t)a;
    dst[e - e0] = (int64_t)b;
  }
}

void xo_er_edges(int64_t n, uint64_t seed, int64_t e0, int64_t e1, int64_t *src, int64_t *dst) {
#pragma omp parallel for schedule(static)
  for (int64_t e = e0; e < e1; e++) {
    src[e - e0] = (int64_t)xo_mulhi(xo_rand(seed, XO_STREAM_ER, 2u * (uint64_t)e), (uint64_t)n);
    dst[e - e0] = (int64_t)xo_mulhi(xo_rand(seed, XO_STREAM_ER, 2u * (uint64_t)e + 1u), (uint64_t)n);
  }
}

int64_t xo_rgg_edges(int64_t n, uint64_t seed, double r2, int64_t cap, int64_t *src, int64_t *dst) {
  const double inv53 = 1.0 / 9007199254740992.0; /* 2^-53 */
  double *x = (double *)malloc(sizeof(double) * (size_t)n), *y = (double *)malloc(sizeof(double) * (size_t)n);
  for (int64_t i = 0; i < n; i++) {
    x[i] = (double)(xo_rand(seed, XO_STREAM_RGG, 2u * (uint64_t)i) >> 11) * inv53;
    y[i] = (double)(xo_rand(seed, XO_STREAM_RGG, 2u * (uint64_t)i + 1u) >> 11) * inv53;
  }
  /* cells no smaller than the radius: every pair within it sits in the same
   * or an adjacent cell, so only those pairs are tested */
  int64_t G = (int64_t)floor(1.0 / (sqrt(r2) * 1.0001));
  if (G < 1) G = 1;
  if (G > 4096) G = 4096;
  int64_t *cstart = (int64_t *)calloc((size_t)(G * G + 1), sizeof(int64_t));
  int64_t *order = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
  int64_t *cell = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
  for (int64_t i = 0; i < n; i++) {
    int64_t cx = (int64_t)(x[i] * (double)G), cy = (int64_t)(y[i] * (double)G);
    if (cx >= G) cx = G - 1;
    if (cy >= G) cy = G - 1;
    cell[i] = cy * G + cx;
    cstart[cell[i] + 1]++;
  }
  for (int64_t c = 0; c < G * G; c++) cstart[c + 1] += cstart[c];
  {
    int64_t *cur = (int64_t *)malloc(sizeof(int64_t) * (size_t)(G * G));
    memcpy(cur, cstart, sizeof(int64_t) * (size_t)(G * G));
    for (int64_t i = 0; i < n; i++) order[cur[cell[i]]++] = i;
    free(cur);
  }
  int64_t cnt = 0;
  for (int64_t u = 0; u < n; u++) {
    int64_t cx = cell[u] % G, cy = cell[u] / G;
    for (int64_t dy = -1; dy <= 1; dy++)
      for (int64_t dx = -1; dx <= 1; dx++) {
        int64_t nx = cx + dx, ny = cy + dy;
        if (nx < 0 || ny < 0 || nx >= G || ny >= G) continue;
        int64_t c = ny * G + nx;
        for (int64_t k = cstart[c]; k < cstart[c + 1]; k++) {
          int64_t v = order[k];
          if (v <= u) continue;
          double ddx = x[u] - x[v], ddy = y[u] - y[v];
          double d2 = ddx * ddx + ddy * ddy;
          if (d2 <= r2) {
            if (cnt < cap) { src[cnt] = u; dst[cnt] = v; }
            cnt++;
          }
        }
      }
  }
  free(x); free(y); free(cstart); free(order); free(cell);
  return cnt <= cap ? cnt : -cnt;
}

/* ======================================================================== */
/* the reference's RGG generator with its parallel LCG, P strips emulated    */
/* ======================================================================== */

uint32_t xo_seed_seq1(uint32_t s) {
  /* std::seed_seq::generate (C++ [rand.util.seedseq]) for one input word
   * and one output word: n=1, t=0, p=0, q=0, m=2 */
  uint32_t b = 0x8b8b8b8bu;
  const uint32_t n = 1;
  for (uint32_t k = 0; k < 2; k++) {
    uint32_t x = b ^ b ^ b; /* b[k%n] ^ b[(k+p)%n] ^ b[(k-1)%n], all the same word */
    uint32_t r1 = 1664525u * (x ^ (x >> 27));
    uint32_t r2 = r1 + (k == 0 ? 1u /* s = size of the seed list */ : (k % n) + s);
    b += r1; /* b[(k+p)%n] += r1 */
    b += r2; /* b[(k+q)%n] += r2 */
    b = r2;  /* b[k%n] = r2 */
  }
  for (uint32_t k = 2; k < 3; k++) {
    uint32_t x = b + b + b;
    uint32_t r3 = 1566083941u * (x ^ (x >> 27));
    uint32_t r4 = r3 - (k % n);
    b ^= r3;
    b ^= r4;
    b = r4;
  }
  return b;
}

typedef struct { int64_t i, j; } xo_pair;

static int xo_pair_cmp(const void *a, const void *b) {
  const xo_pair *x = (const xo_pair *)a, *y = (const xo_pair *)b;
  if (x->i != y->i) return x->i < y->i ? -1 : 1;
  if (x->j != y->j) return x->j < y->j ? -1 : 1;
  return 0;
}

typedef struct { xo_pair *p; int64_t n, cap; } xo_vec;
static void xo_push(xo_vec *v, int64_t i, int64_t j) {
  if (v->n == v->cap) {
    v->cap = v->cap ? 2 * v->cap : 1024;
    v->p = (xo_pair *)realloc(v->p, sizeof(xo_pair) * (size_t)v->cap);
  }
  v->p[v->n].i = i; v->p[v->n].j = j; v->n++;
}

/* 2x2 int64 matrix product with wrap-around, as the reference's unmodded
 * matmat_2x2 (utils.hpp:272-284) computes it */
static void xo_mat2(int64_t c[4], const int64_t a[4], const int64_t b[4]) {
  int64_t t[4];
  for (int i = 0; i < 2; i++)
    for (int j = 0; j < 2; j++) {
      uint64_t s = 0;
      for (int k = 0; k < 2; k++) s += (uint64_t)a[i * 2 + k] * (uint64_t)b[k * 2 + j];
      t[i * 2 + j] = (int64_t)s;
    }
  memcpy(c, t, sizeof(t));
}

int64_t xo_ref_rgg(int64_t nv, int P, double radius, int64_t cap, int64_t *off, int64_t *tails) {
  if (nv <= 0 || P <= 0 || (P & (P - 1)) || nv % P) return -1;
  const int64_t n = nv / P;          /* GenerateRGG::n_ (graph.hpp:767) */
  const int64_t nl = 2 * n;          /* LCG::n_ = 2*n_ (graph.hpp:868) */
  const int64_t MLCG = 2147483647LL; /* deftypes.hpp:14-16 */
  const double PI_REF = 3.14159;     /* deftypes.hpp:7 */
  double rn;
  if (radius > 0) rn = radius;
  else {
    double rc = sqrt((double)log((double)nv) / (double)(PI_REF * (double)nv));
    double rt = sqrt((double)2.0736 / (double)nv);
    rn = (rc + rt) / (double)2.0; /* graph.hpp:788-791 */
  }
  if (!((1.0 / (double)P) > rn)) return -1; /* graph.hpp:793 */

  /* LCG prefix (utils.hpp:310-348): every rank's M^(nl), then a hypercube
   * prefix over ranks, all in wrapping int64 */
  int64_t M[4] = {16807, 0, 0, 1}, Mk[4];
  memcpy(Mk, M, sizeof(M));
  for (int64_t p = 0; p < nl - 1; p++) xo_mat2(Mk, Mk, M); /* mat_power (utils.hpp:294-303) */
  int64_t (*G)[4] = (int64_t(*)[4])malloc(sizeof(int64_t[4]) * (size_t)P);
  int64_t (*R)[4] = (int64_t(*)[4])malloc(sizeof(int64_t[4]) * (size_t)P);
  int64_t (*Pf)[4] = (int64_t(*)[4])malloc(sizeof(int64_t[4]) * (size_t)P);
  for (int r = 0; r < P; r++) {
    memcpy(G[r], Mk, sizeof(Mk));
    Pf[r][0] = 1; Pf[r][1] = 0; Pf[r][2] = 0; Pf[r][3] = 1;
  }
  int steps = 0;
  while ((1 << steps) < P) steps++;
  for (int s = 0; s < steps; s++) {
    for (int r = 0; r < P; r++) memcpy(R[r], G[r ^ (1 << s)], sizeof(int64_t[4]));
    for (int r = 0; r < P; r++) {
      int mate = r ^ (1 << s);
      xo_mat2(G[r], G[r], R[r]);
      if (mate < r) xo_mat2(Pf[r], Pf[r], R[r]);
    }
  }
  const int64_t x0 = (int64_t)xo_seed_seq1(1); /* reseeder(1), utils.hpp:37-44 */
  double *X = (double *)malloc(sizeof(double) * (size_t)(nl * P));
  double *Y = (double *)malloc(sizeof(double) * (size_t)(n * P));
  int64_t *rn64 = (int64_t *)malloc(sizeof(int64_t) * (size_t)nl);
  const double mult = 1.0 / (double)(1.0 + (double)(MLCG - 1));
  const double rec_np = (double)(1.0 / (double)P);
  for (int r = 0; r < P; r++) {
    if (r == 0) rn64[0] = x0;
    else rn64[0] = (int64_t)((uint64_t)x0 * (uint64_t)Pf[r][0] + (uint64_t)Pf[r][2]) % MLCG;
    for (int64_t i = 1; i < nl; i++) rn64[i] = (rn64[i - 1] * 16807 + 0) % MLCG; /* utils.hpp:371-373 */
    double *Xr = X + (size_t)r * (size_t)nl;
    for (int64_t i = 0; i < nl; i++) Xr[i] = (double)((double)fabs((double)rn64[i]) * mult);
    const double lo = r * rec_np, range = (1.0 / (double)P);
    for (int64_t i = n, j = 0; i < nl; i++, j++) Y[(size_t)r * (size_t)n + j] = lo + (double)(range * Xr[i]);
  }
  free(rn64); free(G); free(R); free(Pf);

  /* edges per rank, in the order and with the pair rules of graph.hpp:919-1095 */
  xo_vec *E = (xo_vec *)calloc((size_t)P, sizeof(xo_vec));
  for (int r = 0; r < P; r++) {
    const double *Xr = X + (size_t)r * (size_t)nl, *Yr = Y + (size_t)r * (size_t)n;
    const int64_t base = (int64_t)r * n;
    for (int64_t i = 0; i < n; i++)
      for (int64_t j = i + 1; j < n; j++) {
        double dx = Xr[i] - Xr[j], dy = Yr[i] - Yr[j];
        double ed = sqrt(dx * dx + dy * dy);
        if (ed <= rn) { xo_push(&E[r], i, base + j); xo_push(&E[r], j, base + i); }
      }
    for (int side = 0; side < 2; side++) { /* 0: up (r-1), 1: down (r+1) */
      int q = side == 0 ? r - 1 : r + 1;
      if (q < 0 || q >= P) continue;
      const double *Xq = X + (size_t)q * (size_t)nl, *Yq = Y + (size_t)q * (size_t)n;
      for (int64_t i = 0; i < n; i++)
        for (int64_t j = i + 1; j < n; j++) {
          double dx = Xr[i] - Xq[j], dy = Yr[i] - Yq[j];
          double ed = sqrt(dx * dx + dy * dy);
          if (ed <= rn) {
            xo_push(&E[r], i, (int64_t)q * n + j);
            xo_push(&E[q], j, base + i);
          }
        }
    }
  }
  free(X); free(Y);
  int64_t total = 0;
  for (int r = 0; r < P; r++) total += E[r].n;
  if (total > cap) {
    for (int r = 0; r < P; r++) free(E[r].p);
    free(E);
    return -total;
  }
  int64_t pos = 0;
  off[0] = 0;
  for (int r = 0; r < P; r++) {
    qsort(E[r].p, (size_t)E[r].n, sizeof(xo_pair), xo_pair_cmp); /* graph.hpp:1306-1314 */
    int64_t k = 0;
    for (int64_t i = 0; i < n; i++) {
      while (k < E[r].n && E[r].p[k].i == i) tails[pos++] = E[r].p[k++].j;
      off[(int64_t)r * n + i + 1] = pos;
    }
    free(E[r].p);
  }
  free(E);
  return total;
}

/* ======================================================================== */
/* the batch workload (twin of xt_batch_spec / xt_gen_batch)                */
/* ======================================================================== */

#define XO_STREAM_BATCH 5

void xo_batch_spec(int64_t ng, uint64_t seed, int32_t *kind, int64_t *n, double *mean_deg, uint64_t *gseed) {
  for (int64_t i = 0; i < ng; i++) {
    const uint64_t r0 = xo_rand(seed, XO_STREAM_BATCH, 4u * (uint64_t)i);
    const uint64_t r1 = xo_rand(seed, XO_STREAM_BATCH, 4u * (uint64_t)i + 1u);
    const uint64_t r2 = xo_rand(seed, XO_STREAM_BATCH, 4u * (uint64_t)i + 2u);
    const uint64_t r3 = xo_rand(seed, XO_STREAM_BATCH, 4u * (uint64_t)i + 3u);
    kind[i] = (int32_t)(i & 1);
    const uint64_t oct = r0 >> 61, base = (uint64_t)256 << oct;
    n[i] = (int64_t)(base + xo_mulhi(r1, base));
    const uint64_t doct = xo_mulhi(r2, 3u);
    mean_deg[i] = (double)((uint64_t)8 << doct) * (1.0 + (double)(r3 >> 11) * (1.0 / 9007199254740992.0));
    gseed[i] = xo_mix64(seed ^ (0x9e3779b97f4a7c15ULL * (uint64_t)(i + 1)));
  }
}

/* one graph of the batch: returns its edge count (u,v local ids) or
 * -(needed) when cap is too small */
int64_t xo_batch_graph(int32_t kind, int64_t n, double mean_deg, uint64_t gseed, int64_t cap, int64_t *src,
                       int64_t *dst) {
  if (kind == 1) {
    const int64_t m = (int64_t)llround((double)n * mean_deg / 2.0);
    if (m > cap) return -m;
    xo_er_edges(n, gseed, 0, m, src, dst);
    return m;
  }
  const double r2 = mean_deg / (3.14159265358979323846 * (double)n);
  return xo_rgg_edges(n, gseed, r2, cap, src, dst);
}
