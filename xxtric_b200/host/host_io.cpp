// Host-side graph input for the counter: the vite binary format reader and
// writer, and the reference's random-geometric-graph generator with its
// parallel LCG. No device code; these run on the CPU before the CSR is
// handed to the device builder.
#include <stdint.h>
#include <stdio.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <unordered_set>
#include <vector>

#include "../../include/xtric.h"

namespace {

struct File {
  FILE *f = nullptr;
  explicit File(FILE *p) : f(p) {}
  ~File() {
    if (f) fclose(f);
  }
};

bool read_all(FILE *f, void *dst, size_t bytes) {
  char *p = static_cast<char *>(dst);
  while (bytes) {
    size_t k = fread(p, 1, bytes, f);
    if (k == 0) return false;
    p += k;
    bytes -= k;
  }
  return true;
}

// splitmix64 output function and the counter-based stream used by every
// generator of this library
uint64_t mix64(uint64_t z) {
  z ^= z >> 30;
  z *= 0xbf58476d1ce4e5b9ULL;
  z ^= z >> 27;
  z *= 0x94d049bb133111ebULL;
  z ^= z >> 31;
  return z;
}
uint64_t crand(uint64_t seed, uint64_t stream, uint64_t ctr) {
  uint64_t k = mix64(seed * 0x9e3779b97f4a7c15ULL + stream + 0x632be59bd9b4e019ULL);
  return mix64(k ^ (ctr * 0x9e3779b97f4a7c15ULL + 0xd1b54a32d192ed03ULL));
}
uint64_t mulhi(uint64_t a, uint64_t b) { return uint64_t((unsigned __int128)a * b >> 64); }

}  // namespace

extern "C" {

xt_status xt_vite_read(const char *path, int elem_bytes, int64_t *nv, int64_t *ne, int64_t *offsets,
                       int64_t *tails) {
  if (!path || !nv || !ne || (elem_bytes != 8 && elem_bytes != 4)) return XT_ERR_INVALID;
  File f(fopen(path, "rb"));
  if (!f.f) return XT_ERR_IO;
  int64_t hdr[2];
  if (elem_bytes == 8) {
    if (!read_all(f.f, hdr, sizeof(hdr))) return XT_ERR_IO;
  } else {
    int32_t h32[2];
    if (!read_all(f.f, h32, sizeof(h32))) return XT_ERR_IO;
    hdr[0] = h32[0];
    hdr[1] = h32[1];
  }
  if (hdr[0] < 0 || hdr[1] < 0) return XT_ERR_IO;
  // the file must hold exactly the header, nv+1 offsets and ne records
  if (fseeko(f.f, 0, SEEK_END) != 0) return XT_ERR_IO;
  const int64_t size = ftello(f.f);
  const int64_t want = 2 * elem_bytes + (hdr[0] + 1) * elem_bytes + hdr[1] * 2 * elem_bytes;
  if (size != want) return XT_ERR_IO;
  *nv = hdr[0];
  *ne = hdr[1];
  if (!offsets) return XT_OK;  // sizing call
  if (fseeko(f.f, 2 * elem_bytes, SEEK_SET) != 0) return XT_ERR_IO;
  const int64_t n = hdr[0], m = hdr[1];
  if (elem_bytes == 8) {
    if (!read_all(f.f, offsets, sizeof(int64_t) * (n + 1))) return XT_ERR_IO;
  } else {
    std::vector<int32_t> o(n + 1);
    if (!read_all(f.f, o.data(), sizeof(int32_t) * (n + 1))) return XT_ERR_IO;
    for (int64_t i = 0; i <= n; i++) offsets[i] = o[i];
  }
  if (offsets[0] != 0 || offsets[n] != m) return XT_ERR_IO;
  for (int64_t i = 0; i < n; i++)
    if (offsets[i + 1] < offsets[i]) return XT_ERR_IO;
  // records {tail, weight}; weights are read past (the count ignores them)
  const int64_t chunk = int64_t(1) << 20;
  std::vector<char> buf(size_t(chunk) * 2 * elem_bytes);
  for (int64_t e = 0; e < m; e += chunk) {
    const int64_t k = std::min(chunk, m - e);
    if (!read_all(f.f, buf.data(), size_t(k) * 2 * elem_bytes)) return XT_ERR_IO;
    for (int64_t i = 0; i < k; i++) {
      if (elem_bytes == 8) {
        int64_t t;
        std::memcpy(&t, buf.data() + i * 16, 8);
        tails[e + i] = t;
      } else {
        int32_t t;
        std::memcpy(&t, buf.data() + i * 8, 4);
        tails[e + i] = t;
      }
    }
  }
  return XT_OK;
}

xt_status xt_vite_write(const char *path, int elem_bytes, int64_t nv, const int64_t *offsets,
                        const int64_t *tails) {
  if (!path || nv < 0 || !offsets || (elem_bytes != 8 && elem_bytes != 4)) return XT_ERR_INVALID;
  const int64_t m = offsets[nv];
  if (m > 0 && !tails) return XT_ERR_INVALID;
  File f(fopen(path, "wb"));
  if (!f.f) return XT_ERR_IO;
  auto put = [&](const void *p, size_t b) { return fwrite(p, 1, b, f.f) == b; };
  if (elem_bytes == 8) {
    int64_t hdr[2] = {nv, m};
    if (!put(hdr, sizeof(hdr)) || !put(offsets, sizeof(int64_t) * (nv + 1))) return XT_ERR_IO;
    std::vector<char> rec(16);
    const double w = 1.0;
    for (int64_t e = 0; e < m; e++) {
      std::memcpy(rec.data(), &tails[e], 8);
      std::memcpy(rec.data() + 8, &w, 8);
      if (!put(rec.data(), 16)) return XT_ERR_IO;
    }
  } else {
    if (nv > INT32_MAX || m > INT32_MAX) return XT_ERR_OVERFLOW;
    int32_t hdr[2] = {int32_t(nv), int32_t(m)};
    if (!put(hdr, sizeof(hdr))) return XT_ERR_IO;
    for (int64_t i = 0; i <= nv; i++) {
      int32_t o = int32_t(offsets[i]);
      if (!put(&o, 4)) return XT_ERR_IO;
    }
    const float w = 1.0f;
    for (int64_t e = 0; e < m; e++) {
      int32_t t = int32_t(tails[e]);
      if (!put(&t, 4) || !put(&w, 4)) return XT_ERR_IO;
    }
  }
  return XT_OK;
}

// Tab-separated edge lists as the reference's cuGraph comparison reads them
// (cugraph/cug_triangle_count.py:23-26: columns src, dst, weight; ids used
// as given, renumber=False, so nv = largest id + 1). Blank lines and lines
// starting with '#' or '%' are skipped; a third column is read past and
// ignored. Ids must be integers in [0, 2^31 - 1).
xt_status xt_tsv_read(const char *path, int64_t *nv, int64_t *ne, int32_t *src, int32_t *dst, int64_t cap) {
  if (!path || !nv || !ne) return XT_ERR_INVALID;
  File f(fopen(path, "rb"));
  if (!f.f) return XT_ERR_IO;
  std::vector<char> buf(size_t(1) << 20);
  std::string carry;
  int64_t rows = 0, maxid = -1;
  bool bad = false;
  auto line = [&](const char *a, const char *b) {
    while (a < b && (*a == ' ' || *a == '\t')) a++;
    if (a == b || *a == '#' || *a == '%' || *a == '\r') return;
    int64_t v[2];
    for (int k = 0; k < 2; k++) {
      while (a < b && (*a == ' ' || *a == '\t')) a++;
      if (a == b || *a < '0' || *a > '9') {
        bad = true;
        return;
      }
      int64_t x = 0;
      while (a < b && *a >= '0' && *a <= '9') {
        x = x * 10 + (*a - '0');
        if (x >= INT32_MAX) {
          bad = true;
          return;
        }
        a++;
      }
      v[k] = x;
    }
    if (a < b && *a != '\t' && *a != ' ' && *a != '\r') {
      bad = true;
      return;
    }
    if (src) {
      if (rows >= cap) {
        bad = true;
        return;
      }
      src[rows] = int32_t(v[0]);
      dst[rows] = int32_t(v[1]);
    }
    maxid = std::max(maxid, std::max(v[0], v[1]));
    rows++;
  };
  size_t k;
  while (!bad && (k = fread(buf.data(), 1, buf.size(), f.f)) > 0) {
    const char *p = buf.data(), *end = p + k;
    while (!bad) {
      const char *nl = static_cast<const char *>(memchr(p, '\n', size_t(end - p)));
      if (!nl) {
        carry.append(p, end);
        break;
      }
      if (!carry.empty()) {
        carry.append(p, nl);
        line(carry.data(), carry.data() + carry.size());
        carry.clear();
      } else {
        line(p, nl);
      }
      p = nl + 1;
    }
  }
  if (!bad && !carry.empty()) line(carry.data(), carry.data() + carry.size());
  if (bad) return src && rows >= cap ? XT_ERR_OVERFLOW : XT_ERR_IO;
  *ne = rows;
  *nv = maxid + 1;
  return XT_OK;
}

xt_status xt_tsv_write(const char *path, int64_t ne, const int32_t *src, const int32_t *dst) {
  if (!path || ne < 0 || (ne > 0 && (!src || !dst))) return XT_ERR_INVALID;
  File f(fopen(path, "wb"));
  if (!f.f) return XT_ERR_IO;
  for (int64_t i = 0; i < ne; i++)
    if (fprintf(f.f, "%d\t%d\t1\n", src[i], dst[i]) < 0) return XT_ERR_IO;
  return XT_OK;
}

// The reference's random geometric graph (graph.hpp:745-1364) generated by
// nprocs emulated strip ranks with the LCG of utils.hpp:245-430.
//
// Geometry and RNG follow the reference bit for bit: r(n) with PI = 3.14159
// (deftypes.hpp:7, graph.hpp:788-791); the LCG x <- 16807 x mod (2^31-1)
// seeded by std::seed_seq({1}) (utils.hpp:37-44, 261); the per-rank jump by
// a hypercube prefix of 2x2 matrix powers computed without modulus in
// wrapping int64 (utils.hpp:272-348); X = the first n/p doubles of a rank's
// 2n/p, Y = the rest rescaled into the rank's strip (utils.hpp:399-421); an
// edge when sqrt(dx*dx+dy*dy) <= r (graph.hpp:919-948); cross-strip pairs
// only between adjacent strips and only when the local indices differ
// (graph.hpp:976-1036). Pairs are found through a grid of cells no smaller
// than r instead of the reference's all-pairs loops; the predicate applied to
// each candidate pair is the same expression, so the edge set is identical.
//
// random_edge_pct > 0 adds the reference's extra random edges (graph.hpp:
// 1099-1283) with the same counts and rules, drawn from the seeded counter
// RNG: the reference seeds that step from time(0)^getpid() (graph.hpp:1151),
// so its output is not reproducible; and its per-rank share is left
// uninitialised when nrande < nprocs (graph.hpp:1108-1113), zero here.
// Rows are sorted like the reference's (graph.hpp:1306-1341); duplicates that
// the random step can create are kept, as the reference keeps them.
}  // extern "C"

// The reference's set-up of its random geometric graph for P strip ranks
// (the host part of graph.hpp:745-1364 and utils.hpp:245-430): the radius
// r(n) with PI = 3.14159 (deftypes.hpp:7, graph.hpp:788-791) unless radius >
// 0 is given; the LCG seed std::seed_seq({1}) (utils.hpp:37-44, 261); each
// rank's first LCG value, jumped ahead by a hypercube prefix of 2x2 matrix
// powers computed without modulus in wrapping int64 (utils.hpp:272-348);
// each rank's strip [lo, lo + range) (utils.hpp:399-421). Shared by the host
// generator below and the device generator (csrc/rgg.cu).
xt_status xt_rgg_setup(int64_t nv, int nprocs, double radius, double *rn_out, int64_t *x0, double *lo,
                       double *range) {
  if (nv <= 0 || nprocs <= 0 || (nprocs & (nprocs - 1)) || nv % nprocs) return XT_ERR_INVALID;
  const int P = nprocs;
  const int64_t n = nv / P, nl = 2 * n;
  const int64_t MLCG = 2147483647LL;
  const double PI_REF = 3.14159;
  double rn;
  if (radius > 0) rn = radius;
  else {
    double rc = std::sqrt(double(std::log(double(nv))) / double(PI_REF * double(nv)));
    double rt = std::sqrt(double(2.0736) / double(nv));
    rn = (rc + rt) / double(2.0);
  }
  if (!((1.0 / double(P)) > rn)) return XT_ERR_INVALID;
  // LCG jump-ahead prefix, wrapping int64 like the reference's unmodded
  // 2x2 products
  auto mat2 = [](int64_t c[4], const int64_t a[4], const int64_t b[4]) {
    int64_t t[4];
    for (int i = 0; i < 2; i++)
      for (int j = 0; j < 2; j++) {
        uint64_t s = 0;
        for (int k = 0; k < 2; k++) s += uint64_t(a[i * 2 + k]) * uint64_t(b[k * 2 + j]);
        t[i * 2 + j] = int64_t(s);
      }
    std::memcpy(c, t, sizeof(t));
  };
  const int64_t M[4] = {16807, 0, 0, 1};
  int64_t Mk[4];
  std::memcpy(Mk, M, sizeof(M));
  for (int64_t p = 0; p < nl - 1; p++) mat2(Mk, Mk, M);
  std::vector<std::array<int64_t, 4>> G(P), R(P), Pf(P);
  for (int r = 0; r < P; r++) {
    std::memcpy(G[r].data(), Mk, sizeof(Mk));
    Pf[r] = {1, 0, 0, 1};
  }
  for (int s = 0; (1 << s) < P; s++) {
    for (int r = 0; r < P; r++) R[r] = G[r ^ (1 << s)];
    for (int r = 0; r < P; r++) {
      mat2(G[r].data(), G[r].data(), R[r].data());
      if ((r ^ (1 << s)) < r) mat2(Pf[r].data(), Pf[r].data(), R[r].data());
    }
  }
  std::seed_seq seq({1u});
  uint32_t x0w = 0;
  seq.generate(&x0w, &x0w + 1);
  const int64_t xs = int64_t(x0w);
  const double rec_np = double(1.0 / double(P));
  for (int r = 0; r < P; r++) {
    x0[r] = (r == 0) ? xs : int64_t(uint64_t(xs) * uint64_t(Pf[r][0]) + uint64_t(Pf[r][2])) % MLCG;
    lo[r] = r * rec_np;
  }
  *range = 1.0 / double(P);
  *rn_out = rn;
  return XT_OK;
}

extern "C" {

xt_status xt_rgg_generate(int64_t nv, int nprocs, double radius, double random_edge_pct, uint64_t seed,
                          int64_t cap, int64_t *ne, int64_t *offsets, int64_t *tails) {
  if (!ne || nv <= 0 || nprocs <= 0 || (nprocs & (nprocs - 1)) || nv % nprocs) return XT_ERR_INVALID;
  if (random_edge_pct < 0.0 || random_edge_pct >= 100.0) return XT_ERR_INVALID;
  const int P = nprocs;
  const int64_t n = nv / P, nl = 2 * n;
  const int64_t MLCG = 2147483647LL;
  double rn = 0, range = 0;
  std::vector<int64_t> x0s(P);
  std::vector<double> los(P);
  if (xt_rgg_setup(nv, P, radius, &rn, x0s.data(), los.data(), &range) != XT_OK) return XT_ERR_INVALID;
  std::vector<double> X(size_t(n) * P), Y(size_t(n) * P);
  {
    std::vector<int64_t> rnum(nl);
    const double mult = 1.0 / double(1.0 + double(MLCG - 1));
    std::vector<double> drand(nl);
    for (int r = 0; r < P; r++) {
      rnum[0] = x0s[r];
      for (int64_t i = 1; i < nl; i++) rnum[i] = (rnum[i - 1] * 16807 + 0) % MLCG;
      for (int64_t i = 0; i < nl; i++) drand[i] = double(double(std::fabs(double(rnum[i]))) * mult);
      const double lo = los[r];
      for (int64_t i = 0; i < n; i++) {
        X[size_t(r) * n + i] = drand[i];
        Y[size_t(r) * n + i] = lo + double(range * drand[n + i]);
      }
    }
  }
  // candidate pairs from a grid of cells no smaller than r
  int64_t Gc = int64_t(std::floor(1.0 / (rn * 1.0001)));
  Gc = std::max<int64_t>(1, std::min<int64_t>(Gc, 8192));
  auto cell_of = [&](double v) {
    int64_t c = int64_t(v * double(Gc));
    return std::max<int64_t>(0, std::min<int64_t>(c, Gc - 1));
  };
  std::vector<int64_t> cstart(static_cast<size_t>(Gc * Gc + 1), 0);
  std::vector<int64_t> order(static_cast<size_t>(nv)), cell(static_cast<size_t>(nv));
  for (int64_t a = 0; a < nv; a++) {
    cell[a] = cell_of(Y[a]) * Gc + cell_of(X[a]);
    cstart[cell[a] + 1]++;
  }
  for (int64_t c = 0; c < Gc * Gc; c++) cstart[c + 1] += cstart[c];
  {
    std::vector<int64_t> cur(cstart.begin(), cstart.end() - 1);
    for (int64_t a = 0; a < nv; a++) order[cur[cell[a]]++] = a;
  }
  std::vector<std::pair<int64_t, int64_t>> E;
  for (int64_t a = 0; a < nv; a++) {
    const int64_t ra = a / n, ia = a % n, cx = cell[a] % Gc, cy = cell[a] / Gc;
    for (int64_t dy = -1; dy <= 1; dy++)
      for (int64_t dx = -1; dx <= 1; dx++) {
        const int64_t nx = cx + dx, ny = cy + dy;
        if (nx < 0 || ny < 0 || nx >= Gc || ny >= Gc) continue;
        const int64_t c = ny * Gc + nx;
        for (int64_t k = cstart[c]; k < cstart[c + 1]; k++) {
          const int64_t b = order[k];
          if (b <= a) continue;
          const int64_t rb = b / n, ib = b % n;
          if (rb != ra) {
            if (rb - ra != 1 && ra - rb != 1) continue;  // only adjacent strips exchange ghosts
            if (ia == ib) continue;                      // j > i on both sides drops equal indices
          }
          const double ddx = X[a] - X[b], ddy = Y[a] - Y[b];
          const double ed = std::sqrt(ddx * ddx + ddy * ddy);
          if (ed <= rn) {
            E.emplace_back(a, b);
            E.emplace_back(b, a);
          }
        }
      }
  }
  if (random_edge_pct > 0.0) {
    // graph.hpp:1099-1283 with a seeded RNG: the per-rank share, the local
    // index test (i == j is skipped even across ranks) and the duplicate test
    // against the rank's own list as the reference makes them
    const int64_t tot_pnedges = int64_t(E.size()) / 2;
    const int64_t nrande = int64_t(random_edge_pct * double(tot_pnedges)) / 100;
    std::vector<std::unordered_set<uint64_t>> own(P);
    for (auto &e : E) own[e.first / n].insert(uint64_t(e.first % n) << 32 | uint64_t(e.second));
    std::vector<std::pair<int64_t, int64_t>> add;
    for (int r = 0; r < P; r++) {
      int64_t pn;
      if (nrande < P) pn = (r == P - 1) ? nrande : 0;
      else pn = nrande / P + ((r == P - 1) ? nrande % P : 0);
      for (int64_t k = 0; k < pn; k++) {
        const int64_t i = int64_t(mulhi(crand(seed, 16 + r, 2 * uint64_t(k)), uint64_t(n)));
        const int64_t gj = int64_t(mulhi(crand(seed, 16 + r, 2 * uint64_t(k) + 1), uint64_t(nv)));
        const int64_t target = gj / n, j = gj % n;
        if (i == j) continue;
        const uint64_t key = uint64_t(i) << 32 | uint64_t(gj);
        if (own[r].count(key)) continue;
        own[r].insert(key);
        const int64_t gi = int64_t(r) * n + i;
        add.emplace_back(gi, gj);
        add.emplace_back(target * n + j, gi);
      }
    }
    E.insert(E.end(), add.begin(), add.end());
  }
  std::sort(E.begin(), E.end());
  *ne = int64_t(E.size());
  if (!offsets) return XT_OK;  // sizing call
  if (cap < int64_t(E.size()) || !tails) return XT_ERR_INVALID;
  std::fill(offsets, offsets + nv + 1, 0);
  for (size_t e = 0; e < E.size(); e++) {
    offsets[E[e].first + 1]++;
    tails[e] = E[e].second;
  }
  for (int64_t i = 0; i < nv; i++) offsets[i + 1] += offsets[i];
  return XT_OK;
}

}  // extern "C"
