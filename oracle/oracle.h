/*
 * CPU oracle -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference algorithms on the counting path, used
 * as the checker by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg.  The product library never links, loads or calls it.
 *
 * Parity pins: this restatement is checked against the reference's own code
 * compiled in place (oracle/_ref: src/Graph.cpp pipeline + cpuTriCount,
 * include/ops/Search.cuh host templates) through the golden vectors in
 * tests/golden/.  4-cycle and 4-clique counts have no reference
 * implementation (rectCountHom is declared only,
 * include/kernels/GraphQueryHom.cuh:48): those are pinned by closed-form
 * known answers only.
 */
#ifndef GARY_ORACLE_H
#define GARY_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Symmetric sorted CSR from an undirected edge list: self loops dropped,
 * duplicates (in either direction) merged.  idx must hold 2*m entries, ptr
 * n+1.  Returns nnz (= 2 * unique undirected edges). */
int64_t orc_sym_csr(uint32_t n, int64_t m, const uint32_t *src, const uint32_t *dst,
                    uint64_t *ptr, uint32_t *idx);

/* Orient a symmetric CSR.  by_degree = 0: keep (u,v) with u > v, the
 * reference's orientation (src/Graph.cpp:34-61); by_degree = 1: keep (u,v)
 * with (deg u, u) < (deg v, v).  Caller ids are kept.  out_idx holds nnz/2. */
void orc_orient(uint32_t n, const uint64_t *ptr, const uint32_t *idx, int by_degree,
                uint64_t *out_ptr, uint32_t *out_idx);

/* cpuTriCount (test/TriQueryTest.cu:17-37) on an oriented CSR, with uint64
 * accumulators (the reference's are unsigned and truncate above 2^32). */
uint64_t orc_tri_count(uint32_t n, const uint64_t *ptr, const uint32_t *idx, int threads);

/* 4-cliques on an oriented CSR: sum over (u,v) in E+ and w in S = N+(u)&N+(v)
 * of |S & N+(w)|. */
uint64_t orc_k4_count(uint32_t n, const uint64_t *ptr, const uint32_t *idx, int threads);

/* Non-induced 4-cycles on a symmetric CSR, each once: for every vertex u of
 * highest rank (degree, id) in the cycle, sum over w of C(c(u,w), 2) where
 * c counts lower-ranked common neighbours. */
uint64_t orc_c4_count(uint32_t n, const uint64_t *ptr, const uint32_t *idx, int threads);

/* tr(A^4) = sum over u,w of (A^2)_{uw}^2 on a symmetric CSR (hom(C4)); O(n d^2). */
uint64_t orc_c4_hom(uint32_t n, const uint64_t *ptr, const uint32_t *idx);

/* Algorithmic byte count of the triangle pass on an oriented CSR:
 * sum over (u,v) in E+ of 4(d+(u) + d+(v)) + 24; also the wedge total. */
void orc_tc_bytes(uint32_t n, const uint64_t *ptr, const uint32_t *idx, uint64_t *wedges,
                  uint64_t *alg_bytes);

/* std::set_intersection semantics (test/SetOpTest.cu:94-96). */
int64_t orc_intersect(const uint32_t *a, int64_t na, const uint32_t *b, int64_t nb,
                      uint32_t *out /* may be NULL: count only */);

/* orc_intersect over a batch of pairs, OpenMP over pairs; counts may be NULL. */
uint64_t orc_intersect_batch(int64_t npairs, const int64_t *a_off, const int32_t *la,
                             const uint32_t *a, const int64_t *b_off, const int32_t *lb,
                             const uint32_t *b, int64_t *counts, int threads);

/* binary_search (include/ops/Search.cuh:48-61) */
int orc_binary_search(const uint32_t *list, int64_t n, uint32_t key);
/* build_cache (Search.cuh:93-100): cache[i] = list[i*n/N], 64-bit index math */
void orc_build_cache(const uint32_t *list, int64_t n, int N, uint32_t *cache);
/* binary_search_2phase (Search.cuh:120-138) */
int orc_binary_search_2phase(const uint32_t *list, int64_t n, const uint32_t *cache, int N,
                             uint32_t key);

/* Cost-model network (6 -> 64 -> 64 -> 4, ReLU), FP64 restatement of the
 * GPU kernels for gradient checks.  `params` uses the GPU block layout
 * (20 normalisation floats, then W1, b1, W2, b2, W3, b3).  orc_mlp_grad
 * returns d(loss)/d(weights) for loss = sum over masked cells of
 * (y - t)^2 / norm, in standardised units, into grad[4888] (normalisation
 * entries zero), and the unnormalised squared-error sum in *loss. */
void orc_mlp_forward(const float *params, const float *x, int64_t n, double *y);
void orc_mlp_grad(const float *params, const float *x, const float *t, const uint8_t *mask,
                  int64_t n, double norm, double *grad, double *loss);

/* ---- the synthetic workload, restated for the reference arm ------------
 * bench.py's reference arm must build its input without the product library,
 * so the seeded RMAT generator (a workload definition of this project, not a
 * reference algorithm) is restated here: counter-based splitmix64 draws,
 * (a,b,c,d) = (.57,.19,.19,.05) by integer thresholds floor(2^32 *
 * {.57,.76,.95}), two levels per 64-bit draw, no noise, no permutation.
 * tests/test_oracle.py checks it edge for edge against gary_gen_rmat. */
void orc_gen_rmat(int scale, uint64_t seed, uint64_t first, uint64_t count, uint32_t *src,
                  uint32_t *dst);

/* Unique undirected edges of an edge list over [0, n): self loops dropped,
 * duplicates in either direction merged, each edge written once as
 * (us[k], vs[k]) with us[k] < vs[k], sorted by (u, v).  us and vs hold m
 * entries.  Returns the number written.  OpenMP over rows. */
int64_t orc_unique_edges(uint32_t n, int64_t m, const uint32_t *src, const uint32_t *dst,
                         uint32_t *us, uint32_t *vs, int threads);

#ifdef __cplusplus
}
#endif
#endif
