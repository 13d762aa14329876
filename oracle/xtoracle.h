/*
 * xtoracle — CPU restatement of sg0/xxtric's counting path and of the graph
 * generators, used ONLY as the checker for the CUDA product (tests, smoke,
 * and the CPU-baseline leg of bench.py). Nothing in the product links it.
 *
 * Parity pins: counts agree with the reference's own unmodified CPU binary
 * (oracle/_ref/tric, built from main.cpp + graph.hpp + utils.hpp + xxtric.hpp
 * against mpi_shim/mpi.h) on every golden fixture under tests/golden/.
 */
#ifndef XTORACLE_H
#define XTORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- counting --------------------------------------------------------- */

/* The reference's single-rank count: erange build (xxtric.hpp:60-80), the
 * local loop (xxtric.hpp:150-207), check_edgelist (xxtric.hpp:516-545) and
 * the min/max prunes (xxtric.hpp:576-588), on a CSR of nv vertices whose
 * rows are sorted (the reference's trusted-input contract). */
int64_t xo_count_xxtric(int64_t nv, const int64_t *off, const int64_t *tails);

/* Independent counter: id-oriented sorted merge over a canonical (sorted,
 * deduped, symmetric, loop-free) CSR. Credits all three corners of every
 * triangle into per_vertex (nullable), the cuGraph convention
 * (cugraph/cug_triangle_count.py:33-41). OpenMP-parallel. */
int64_t xo_count_merge(int64_t nv, const int64_t *off, const int64_t *tails, int64_t *per_vertex);

/* Per-vertex triangle counts of a few selected vertices of a canonical CSR:
 * the number of edges among N(s), by merging N(s) with N(v), v in N(s). */
void xo_local_counts(int64_t nv, const int64_t *off, const int64_t *tails, int64_t nsel, const int64_t *sel,
                     int64_t *out);

/* ---- canonical CSR ----------------------------------------------------- */

/* Canonicalise an edge list (any id width via int64 arrays): drop self loops,
 * symmetrise, sort and dedup. Writes off[nv+1]; tails must hold 2*ne.
 * Returns the number of directed entries, or -1 on an id outside [0,nv). */
int64_t xo_canon_csr(int64_t nv, int64_t ne, const int64_t *src, const int64_t *dst, int64_t *off,
                     int64_t *tails);

/* ---- deterministic counter-based RNG (shared by every generator) -------- */
uint64_t xo_mix64(uint64_t z);
uint64_t xo_rand(uint64_t seed, uint64_t stream, uint64_t ctr);
/* bijective pseudo-random permutation of [0, 2^bits) */
uint64_t xo_perm(uint64_t x, int bits, uint64_t seed);

/* ---- generators (bit-exact twins of the GPU generators) ----------------- */

/* R-MAT edges [e0,e1) of a 2^scale graph, quadrant weights a,b,c,d in
 * 1/65536 units with per-level multiplicative noise of +-noise_pct percent,
 * ids permuted by xo_perm when permute != 0. */
void xo_rmat_edges(int scale, uint64_t seed, int a16, int b16, int c16, int noise_pct, int permute, int64_t e0,
                   int64_t e1, int64_t *src, int64_t *dst);

/* Chung-Lu edges [e0,e1): endpoints drawn from the integer CDF cdf[0..n]
 * (cdf[0]=0, strictly non-decreasing), ids permuted when permute != 0
 * (n must then be a power of two). */
void xo_chunglu_edges(int64_t n, const uint64_t *cdf, uint64_t seed, int permute, int64_t e0, int64_t e1,
                      int64_t *src, int64_t *dst);

/* Chung-Lu integer weight CDF for n vertices, exponent gamma, mean degree
 * and max expected degree (writes n+1 entries). Returns the edge count m. */
int64_t xo_chunglu_cdf(int64_t n, double gamma, double mean_deg, double max_deg, uint64_t *cdf);

/* Erdos-Renyi G(n, M) edges [e0,e1): uniform ordered pairs. */
void xo_er_edges(int64_t n, uint64_t seed, int64_t e0, int64_t e1, int64_t *src, int64_t *dst);

/* Unit-square random geometric graph: n points from the counter RNG, an
 * edge for every pair with dx*dx+dy*dy <= r2. Writes u<v pairs; returns the
 * count, or -(needed) when cap is too small. */
int64_t xo_rgg_edges(int64_t n, uint64_t seed, double r2, int64_t cap, int64_t *src, int64_t *dst);

/* The reference's RGG generator (graph.hpp:745-1364) with its LCG
 * (utils.hpp:245-430) emulating P strip ranks: returns the directed entry
 * count and fills off[nv+1]/tails (cap entries) in the order the reference
 * builds them. radius <= 0 selects the reference's r(n) (graph.hpp:788-791).
 * Returns -(needed) when cap is too small, -1 on invalid arguments. */
int64_t xo_ref_rgg(int64_t nv, int P, double radius, int64_t cap, int64_t *off, int64_t *tails);

/* std::seed_seq({s}).generate() of one 32-bit word (utils.hpp:37-44) */
uint32_t xo_seed_seq1(uint32_t s);

/* the batch workload: per-graph kind (0 geometric, 1 Erdos-Renyi), size,
 * mean degree and seed; and one graph's edges (local ids; returns the count
 * or -(needed) when cap is too small) */
void xo_batch_spec(int64_t ng, uint64_t seed, int32_t *kind, int64_t *n, double *mean_deg, uint64_t *gseed);
int64_t xo_batch_graph(int32_t kind, int64_t n, double mean_deg, uint64_t gseed, int64_t cap, int64_t *src,
                       int64_t *dst);

#ifdef __cplusplus
}
#endif
#endif
