/*
 * gary_b200.h -- C ABI of the B200 subgraph-counting path.
 *
 * The reference (hirayaku/Gary) exposes this path only as C++ templates:
 *   - DeviceGraphCtx / DeviceCSR / DeviceCOO / DeviceGraph
 *       (include/DeviceGraph.cuh:15-133, src/DeviceGraph.cu:14-96)
 *   - graph_query::triangleCountHom / triangleCountLegacy / getIndexCacheSMem
 *       (include/kernels/GraphQueryHom.cuh:13-48, src/GraphQueryHom.cu:11-38)
 *   - the warp-cooperative set operations of include/ops/{Search,Intersection}.cuh
 * Each entry point below names the reference interface it replaces.  The C++
 * shims in include/gary/ keep the reference's names on top of this ABI.
 *
 * Conventions
 *   - every function returns an int status: GARY_OK (0) or a negative
 *     GARY_ERR_* class; gary_last_error() describes the last failure of the
 *     calling thread.  No C++ exception crosses this boundary.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default
 *     stream).  Calls that return a host value synchronise that stream.
 *   - vertex ids are uint32 (< 2^32 - 1; UINT32_MAX is the list padding
 *     sentinel), edge offsets uint64.  The reference uses int32 / int64
 *     (include/Defines.h:9-10); for every id below 2^31 the order and the
 *     arithmetic are the same.
 *   - a gary_graph is used by one host thread at a time; distinct graphs may
 *     be used concurrently.
 */
#ifndef GARY_B200_H
#define GARY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GARY_ABI_VERSION 2

/* ---- status codes ------------------------------------------------------ */
#define GARY_OK 0
#define GARY_ERR_INVALID (-1)     /* bad argument (null pointer, size, flag) */
#define GARY_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define GARY_ERR_OOM (-3)         /* device or host allocation failed */
#define GARY_ERR_INPUT (-4)       /* malformed graph: unsorted, duplicate, loop, id >= n */
#define GARY_ERR_TIMEOUT (-5)     /* a bounded device wait expired (scheduler, TMA) */
#define GARY_ERR_UNSUPPORTED (-6) /* valid request this build cannot serve */
#define GARY_ERR_INTERNAL (-7)    /* a device table overflowed: a capacity rule was broken */

/* ---- flags for gary_graph_upload / gary_csr_from_edges ----------------- */
#define GARY_INPUT_SYMMETRIC 0x0u /* CSR lists every undirected edge in both rows */
#define GARY_INPUT_DAG 0x1u       /* CSR lists every undirected edge once (any orientation) */
#define GARY_INPUT_DEVICE 0x2u    /* input pointers are device pointers */
#define GARY_KEEP_IDS 0x4u        /* orient by degree but keep caller vertex ids (no relabel) */
#define GARY_VALIDATE 0x8u        /* check sortedness, range and self loops; GARY_ERR_INPUT */

/* ---- patterns and schedulers for gary_count ---------------------------- */
#define GARY_PATTERN_TRIANGLE 3 /* T = sum over oriented edges (u,v) of |N+(u) & N+(v)| */
#define GARY_PATTERN_4CYCLE 4   /* non-induced 4-cycles, each counted once */
#define GARY_PATTERN_4CLIQUE 5  /* 4-cliques, each counted once */

#define GARY_SCHED_PLAIN 0   /* degree-threshold variant dispatch, work-based tile weights */
#define GARY_SCHED_LEARNED 1 /* MLP cost model picks the variant and sets tile weights */

/* ======================================================================== */
const char *gary_last_error(void);
int gary_abi_version(void);

/* ---- device graph: replaces DeviceGraphCtx (include/DeviceGraph.cuh:75-133,
 *      src/DeviceGraph.cu:14-96) ------------------------------------------ */
typedef struct gary_graph gary_graph;

typedef struct gary_graph_info {
  uint32_t n;                /* vertices */
  uint32_t max_degree;       /* max undirected degree */
  uint32_t max_out_degree;   /* max oriented out-degree d+(u) */
  uint32_t relabeled;        /* 1 when vertex ids are degree ranks */
  uint64_t m;                /* undirected edges = |E+| */
  uint64_t adj_words;        /* padded uint32 words of the oriented lists */
  uint64_t wedges;           /* sum over (u,v) in E+ of d+(v) */
  uint64_t out_deg_sq;       /* sum over u of d+(u)^2 */
  uint64_t alg_bytes;        /* B_alg = sum over (u,v) in E+ of 4(d+(u)+d+(v)) + 24 */
  uint64_t device_bytes;     /* bytes of device memory this graph holds */
} gary_graph_info;

/* Raw views with the reference's field names (include/DeviceGraph.cuh:15-67).
 * colIdx + indPtr[v] points at v's oriented list, deg[v] entries long; lists
 * start on 32-byte boundaries and are padded with UINT32_MAX to a multiple of
 * 8 ids.  The COO view has its own unpadded colIdx (the reference aliases the
 * CSR's, DeviceGraph.cuh:117, which padding would break). */
typedef struct gary_device_csr {
  uint32_t m;
  uint64_t nnz;
  const uint64_t *indPtr;
  const uint32_t *colIdx;
  const uint32_t *deg;
} gary_device_csr;

typedef struct gary_device_coo {
  uint32_t m;
  uint64_t nnz;
  const uint32_t *rowIdx;
  const uint32_t *colIdx;
  const uint32_t *deg;
} gary_device_coo;

/* Upload a CSR and build the degree-oriented, 32-byte-aligned, padded uint32
 * lists on the device.  Replaces DeviceGraphCtx::loadFromHost(GraphCSR)
 * (src/DeviceGraph.cu:18-28) plus the host orientation pass
 * (src/Graph.cpp:34-61, convert.cpp:61-78).  Orientation is by (degree, id),
 * not by id: triangle and clique counts do not depend on the order.
 * ptr has n+1 entries, idx has nnz entries; lists sorted ascending, no
 * duplicates, no self loops. */
int gary_graph_upload(const uint64_t *ptr, const uint32_t *idx, uint32_t n, uint64_t nnz,
                      uint32_t flags, void *stream, gary_graph **out);

/* Replaces DeviceGraphCtx::clear() (src/DeviceGraph.cu:54-61). NULL is a no-op. */
int gary_graph_free(gary_graph *g);

int gary_graph_get_info(const gary_graph *g, gary_graph_info *out);

/* Replaces DeviceGraphCtx::getDeviceCSR / getDeviceCOO (include/DeviceGraph.cuh:100-121).
 * The COO arrays are built on first use, like the reference's lazy rowIdx. */
int gary_graph_device_csr(gary_graph *g, gary_device_csr *out);
int gary_graph_device_coo(gary_graph *g, gary_device_coo *out);

/* Host copy of the oriented CSR without padding: ptr[n+1], idx[m].  With
 * relabel on, ids are degree ranks; perm (may be NULL) receives rank -> caller id.
 * Replaces DeviceGraphCtx::getHostCSR (src/DeviceGraph.cu:63-81). */
int gary_graph_download(gary_graph *g, uint64_t *ptr, uint32_t *idx, uint32_t *perm);

/* ---- counting: replaces graph_query::triangleCountHom<useCache,N,Policy>
 *      (include/kernels/GraphQueryHom.cuh:15-43) and triangleCountLegacy
 *      (src/GraphQueryHom.cu:15-38); 4-cycle / 4-clique have no reference
 *      implementation (rectCountHom is declared only, GraphQueryHom.cuh:48). */

/* Count `pattern` and write the uint64 total to *out (host).  Synchronises. */
int gary_count(gary_graph *g, int pattern, int sched, void *stream, uint64_t *out);

/* Same, asynchronous: the total is written to the device word *d_out (which
 * the call zeroes first, unlike the reference, whose caller must zero it,
 * test/TriQueryTest.cu:117).  No host synchronisation.  The launch's own
 * failures (a bounded wait that expired, a table that overflowed) are only
 * known once it has run: gary_count_status reports them. */
int gary_count_async(gary_graph *g, int pattern, int sched, void *stream, uint64_t *d_out);

/* Status of the last counting launch on g (gary_count_async,
 * gary_count_shard_async, gary_batch_count_async or a replay of a captured
 * batch): synchronises `stream` (the launch's stream) and returns GARY_OK,
 * GARY_ERR_TIMEOUT (a bounded device wait expired) or GARY_ERR_INTERNAL (a
 * shared-memory table overflowed); after either error the count on the
 * device is incomplete.  gary_count performs this check itself.  The
 * reference's spins never give up, so it has no counterpart
 * (include/ops/DeviceQueue.cuh:101-108). */
int gary_count_status(gary_graph *g, void *stream);

/* One shard of the count: every rank holds the whole graph and counts tile
 * ranges [shard/nshards, (shard+1)/nshards) of the plan; the shard totals sum
 * to the full count.  No reference counterpart (the reference is single-GPU,
 * src/DeviceGraph.cu:91-96). */
int gary_count_shard_async(gary_graph *g, int pattern, int sched, uint32_t shard,
                           uint32_t nshards, void *stream, uint64_t *d_out);

/* Statistics of the last gary_count* on g (call after its stream is
 * synchronised): kernel time of the counting kernel in milliseconds (CUDA
 * events on its stream), tiles, the triangle kernel's CTA tiles by the
 * shared-memory set that held N+(v) (bitmap of its id span, hash buckets,
 * the list staged whole by a bulk copy, evenly spaced samples for the
 * two-phase search), the launch's error word (0 when it ran clean), and the
 * triangle plan's work: the ids its kernel probes against a set, summed over
 * the whole plan (shards included).  For the triangle kernel also its makespan
 * and the mean time at which its CTAs finished (device clock, from the first
 * CTA start): makespan / mean finish bounds what any other assignment of the
 * same tiles to CTAs could gain.  For benches and tests. */
typedef struct gary_count_stats {
  float kernel_ms;
  uint32_t tiles;
  uint32_t cta_tiles;
  uint32_t cta_path_tiles[4];
  uint32_t error;
  uint64_t work;
  float makespan_ms;
  float mean_cta_finish_ms;
} gary_count_stats;
int gary_count_last_stats(gary_graph *g, gary_count_stats *out);

/* ---- triangle count without device allocation --------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * (all device memory owned by a host framework's pool, or a fixed memory
 * budget): the caller passes an oriented CSR already on the device, in the
 * DeviceCSR layout (indptr[v] = first entry of v, deg[v] = its length; every
 * undirected edge stored once, any acyclic orientation, lists sorted), and a
 * device word for the result.  The library allocates nothing: its only
 * scratch is a 128 KiB file-scope device array that every GPU loading the
 * library holds until exit, and n may be at most 33,550,336 vertices (larger
 * n returns GARY_ERR_INVALID).  The first call on a device looks up that
 * array's device address and should come before any stream capture; the
 * address is kept for the life of the process, so after a cudaDeviceReset
 * (which reloads the module) do not call this entry point again in the same
 * process.  All calls share the array, so calls that overlap on the GPU race;
 * each call clears it before use.  Asynchronous on `stream`. */
int gary_count_triangles_noalloc(const uint64_t *d_indptr, const uint32_t *d_colidx,
                                 const uint32_t *d_deg, uint32_t n, void *stream,
                                 uint64_t *d_out);

/* ---- batches of graphs ---------------------------------------------------
 * Many graphs counted in one persistent launch.  gary_batch_upload takes the
 * disjoint union as one CSR whose vertices [group_off[g], group_off[g+1])
 * form graph g (host offsets, ngroups + 1 entries) and ranks vertices within
 * each graph.  gary_batch_count_async writes the triangle count of every
 * graph to d_counts[g] and their sum to *d_total; the work of all graphs is
 * cut into one tile list fed to the kernel by its device-side queue.
 * gary_batch_capture records that count (queue reset, zeroing, kernel) into a
 * CUDA graph; gary_exec_launch replays it.  No reference counterpart: the
 * reference counts one graph per launch (test/TriQueryTest.cu:114-133). */
typedef struct gary_exec gary_exec;
int gary_batch_upload(const uint64_t *group_off, uint32_t ngroups, const uint64_t *ptr,
                      const uint32_t *idx, uint32_t n, uint64_t nnz, uint32_t flags, void *stream,
                      gary_graph **out);
int gary_batch_count_async(gary_graph *g, int sched, uint64_t *d_counts, uint64_t *d_total,
                           void *stream);
int gary_batch_capture(gary_graph *g, int sched, uint64_t *d_counts, uint64_t *d_total,
                       void *stream, gary_exec **out);
int gary_exec_launch(gary_exec *e, void *stream);
int gary_exec_free(gary_exec *e);

/* Barabasi-Albert graph (seed clique K_{m+1}, m distinct degree-proportional
 * targets per new vertex); edges written once each, *count receives their
 * number (<= m (m+1) / 2 + (n - m - 1) m). */
int gary_gen_ba(uint32_t n, uint32_t m, uint64_t seed, uint32_t *src, uint32_t *dst,
                uint64_t *count);

/* ---- tuning (the autotuner's knobs) -------------------------------------
 * Process-wide parameters of the counting plans, applied to plans built after
 * the call (gary_graph_drop_plans discards a graph's cached plans):
 *   "warp_tile_cost"  target probes per warp tile; 0 (the default) sizes
 *                     it from the graph's work: about 32 tiles per resident
 *                     warp, between 2^11 and 2^15 probes
 *   "cta_tile_cost"   target probes per CTA tile         (default 2^20)
 *   "vertex_overhead" fixed cost charged per vertex      (default 64)
 *   "min_blocks"      resident CTAs per SM, 2 or 3; 0 (the default) picks 3
 *                     from 2^31 probes on, else 2
 *   "warp_cap"        largest out-degree d+(v) a warp's hash set takes
 *                     (8..512, default 512); larger lists whose id span is
 *                     too wide for a warp bitmap go to CTA tiles
 * Two keys change no plan, only how its CTA tiles run, so that small graphs
 * reach every path (tests use them; production leaves them alone):
 *   "cta_set_words"   shared words a CTA tile's set of N+(v) may use: a power
 *                     of two from 64 to 16384, or 0 (the default: all 16384)
 *   "stage_wait_polls" polls of the first wait for a bulk staging copy
 *                     (0..2^24, default 2^24); when it gives up the launch
 *                     reports GARY_ERR_TIMEOUT after draining the copy
 *   "pool_keep_bytes" freed device memory the library keeps for reuse, per
 *                     device and per kind: construction scratch in its
 *                     memory pool across syncs, and the blocks of freed
 *                     graphs and plans (default UINT64_MAX: all of it, like
 *                     a caching allocator, so a repeated upload makes no
 *                     driver allocation call; 0 returns both now and at
 *                     every later free or sync); "reset" leaves it alone
 *   "reset"           restore every plan default
 * No reference counterpart: the reference fixes its launch shape in each test
 * (test/TriQueryTest.cu:98-99, 116-117). */
int gary_tune(const char *key, uint64_t value);
int gary_graph_drop_plans(gary_graph *g);

/* ---- batched set operations: the include/ops layer ---------------------
 * Lists are sorted ascending, values < UINT32_MAX. */
#define GARY_ISECT_AUTO 0   /* SEARCH when 2|L| > |S| log2 |L| (L the longer list), else MERGE */
#define GARY_ISECT_MERGE 1  /* warp merge path over 32-wide windows (ballot / shuffle) */
#define GARY_ISECT_SEARCH 2 /* two-phase search: 256 shared samples, then HBM */
#define GARY_ISECT_BITMAP 3 /* shared bitmap of the longer list over 32K-value windows */

/* |A_i & B_i| for npairs pairs; A_i = d_a[d_a_off[i] .. + d_a_len[i]), B_i likewise.
 * Replaces intersectBinarySearch / intersect (include/ops/Intersection.cuh:18-199)
 * and intersect_bs_cache (Intersection.cuh:240-300), which intersect one pair
 * per warp inside a caller's kernel.  d_counts[i] (optional) receives each
 * count, *d_total (optional) their sum.  With d_out_off set, A_i & B_i is
 * also written, sorted, to d_out + d_out_off[i] (capacity min(|A_i|,|B_i|)).
 * d_queue is one device word of scheduler state owned by the caller. */
int gary_intersect_batch(uint64_t npairs, const uint64_t *d_a_off, const uint32_t *d_a_len,
                         const uint32_t *d_a, const uint64_t *d_b_off, const uint32_t *d_b_len,
                         const uint32_t *d_b, int variant, uint64_t *d_counts,
                         const uint64_t *d_out_off, uint32_t *d_out, uint64_t *d_total,
                         uint64_t *d_queue, void *stream);

/* Bounded and ancestor-filtered counts: the reference's intersect_num family
 * (include/ops/Intersection.cuh:361-485, left commented out there), used by
 * pattern matching with symmetry breaking.  d_counts[i] = the number of x in
 * A_i & B_i with x < d_bound[i] (d_bound NULL: no bound) and x not among the
 * excluded ids d_ex[d_ex_off[i] .. d_ex_off[i+1]) (d_ex_off NULL: none; an id
 * listed twice is excluded once).  Count only; arguments otherwise as
 * gary_intersect_batch. */
int gary_intersect_num_batch(uint64_t npairs, const uint64_t *d_a_off, const uint32_t *d_a_len,
                             const uint32_t *d_a, const uint64_t *d_b_off, const uint32_t *d_b_len,
                             const uint32_t *d_b, int variant, const uint32_t *d_bound,
                             const uint64_t *d_ex_off, const uint32_t *d_ex, uint64_t *d_counts,
                             uint64_t *d_total, uint64_t *d_queue, void *stream);

/* Search nkeys keys in one sorted list (duplicates allowed).  cache_entries = 0:
 * binary_search (include/ops/Search.cuh:48-61); otherwise the two-phase search
 * of Search.cuh:93-138 with that many samples cached per CTA (the reference
 * uses 32; up to 8192).  d_found[i] = 1 when keys[i] is present (optional);
 * *d_count = number present (optional). */
int gary_search_batch(const uint32_t *d_list, uint64_t len, const uint32_t *d_keys, uint64_t nkeys,
                      uint32_t cache_entries, uint8_t *d_found, uint64_t *d_count, void *stream);

/* Set-intersection workload generator (seeded, counter-based; identical on
 * host and device).  gary_zipf_table fills cdf[nmax] with uint64 thresholds
 * of Zipf(s) on [1, nmax] (inverse-CDF sampling; the reference draws Zipf by
 * rejection-inversion, common/Zipf.h:34-172).  Lists of pair i have
 * Zipf lengths and one uniform value per bucket of [0, range); a fraction
 * `overlap` of the shorter list is planted from the longer one.  Device
 * generation is two calls: lengths (and 16-byte-padded quad counts, whose
 * exclusive scan times 4 gives the offsets), then values. */
int gary_zipf_table(uint32_t nmax, double s, uint64_t *cdf);
int gary_gen_pair_host(uint64_t seed, uint64_t pair, uint32_t nmax, const uint64_t *cdf,
                       double overlap, uint64_t range, uint32_t *a, uint32_t *la, uint32_t *b,
                       uint32_t *lb);
int gary_gen_pairs_lengths(uint64_t seed, uint64_t first, uint64_t npairs, uint32_t nmax,
                           const uint64_t *d_cdf, uint32_t *d_la, uint32_t *d_lb, uint64_t *d_qa,
                           uint64_t *d_qb, void *stream);
int gary_gen_pairs_values(uint64_t seed, uint64_t first, uint64_t npairs, uint32_t nmax,
                          const uint64_t *d_cdf, double overlap, uint64_t range,
                          const uint32_t *d_la, const uint32_t *d_lb, const uint64_t *d_a_off,
                          const uint64_t *d_b_off, uint32_t *d_a, uint32_t *d_b, void *stream);

/* ---- learned scheduling: the cost model ---------------------------------
 * A 6 -> 64 -> 64 -> 4 MLP (FP32, ReLU) predicts, for every middle vertex of
 * the triangle kernel, log2 of the cycles each intersection variant (hash,
 * search, regs (at most 8 ids in registers), bitmap: index 0..3) would take.  GARY_SCHED_LEARNED runs
 * every warp vertex with its predicted-cheapest legal variant and cuts tiles
 * by predicted cycles; the plain plan (bitmap when the id span fits, else
 * hash; probe-count tile weights) stays the fallback.  No reference
 * counterpart: the reference has one fixed variant per kernel.
 *
 * Parameter block of gary_mlp_param_count() floats: mu_x[6], sd_x[6],
 * mu_y[4], sd_y[4] (standardisation), then W1[64][6], b1, W2[64][64], b2,
 * W3[4][64], b3.  Training runs on the device: gary_mlp_grad (forward and
 * backward, masked squared error in standardised units) and gary_mlp_adam.
 * Files: "GARYMLP1", uint32 {1, 6, 64, 64, 4}, then the floats. */
int gary_mlp_param_count(void);
int gary_mlp_init(uint64_t seed, float *params);
int gary_mlp_forward(const float *d_params, const float *d_x, uint64_t n, int scale, float *d_y,
                     void *stream);
int gary_mlp_grad(const float *d_params, const float *d_x, const float *d_t, const uint8_t *d_mask,
                  uint64_t n, float norm, float *d_grad, float *d_loss, void *stream);
int gary_mlp_adam(float *d_params, const float *d_grad, float *d_m, float *d_v, uint32_t step,
                  float lr, void *stream);
int gary_mlp_save(const char *path, const float *params);
int gary_mlp_load(const char *path, float *params);
/* Process-wide model for GARY_SCHED_LEARNED (host block; NULL clears). */
int gary_set_cost_model(const float *params);
/* Training data: features d_x[n][6] and legal-variant bits d_legal[n] of every
 * middle vertex (0: not run by a warp), and per-vertex cycles of one run of
 * the triangle kernel with every warp vertex forced to `variant` (-1: plain
 * dispatch).  d_count receives the triangle count (exact for any variant). */
int gary_tc_features(gary_graph *g, float *d_x, uint8_t *d_legal, void *stream);
int gary_tc_profile(gary_graph *g, int variant, uint64_t *d_cycles, uint64_t *d_count,
                    void *stream);

/* ---- symmetric CSR construction on the device ------------------------- *
 * Dedup, drop self loops, symmetrise and sort an undirected edge list into a
 * CSR (the reference does this on the host: src/Graph.cpp:19-32, 63-91). */
typedef struct gary_csr gary_csr;
int gary_csr_from_edges(const uint32_t *src, const uint32_t *dst, uint64_t m, uint32_t n,
                        uint32_t flags, void *stream, gary_csr **out);
int gary_csr_info(const gary_csr *c, uint32_t *n, uint64_t *nnz);
int gary_csr_device_ptrs(const gary_csr *c, const uint64_t **ptr, const uint32_t **idx);
int gary_csr_download(const gary_csr *c, uint64_t *ptr, uint32_t *idx);
int gary_csr_free(gary_csr *c);

/* ---- byte planes -------------------------------------------------------- *
 * Split n words of word_bytes (4 or 8) into word_bytes / plane_bytes planes
 * of plane_bytes (1, 2 or 4, smaller than the word): plane j holds bytes
 * [j * plane_bytes, (j+1) * plane_bytes) of every word, least significant
 * first, in word order.  Replaces the reference's segmentKernel<SrcT, DstT>
 * (include/kernels/SegmentArray.cuh:26-149; its tests, test/CUDATest.cu:60-130).
 * gary_planes_join is the inverse.  d_planes is a HOST array of
 * word_bytes / plane_bytes device pointers; every device pointer must be
 * 16-byte aligned (GARY_ERR_INVALID otherwise).  Asynchronous on `stream`. */
int gary_planes_split(const void *d_words, uint64_t n, int word_bytes, int plane_bytes,
                      void *const *d_planes, void *stream);
int gary_planes_join(void *const *d_planes, uint64_t n, int word_bytes, int plane_bytes, void *d_words,
                     void *stream);

/* ---- the reference's graph binaries (host only, no device use) -------- *
 * Read and write the files the reference saves with cereal's binary archive
 * (GraphCSR / GraphCOO save/load, include/Graph.h:132-148, 269-285; the
 * loadFromBinary / saveToBinary pair, include/Graph.h:300-316; e.g. the
 * csr_dag.bin its tests load, test/TriQueryTest.cu:51).  Layout, little-endian:
 * uint32 version (1), uint32 format (0 CSR, 1 COO), int32 m, int64 nnz, then
 * each array as a cereal shared pointer (uint32 id 0x8000000k) holding a
 * uint64 count and the elements: CSR ptr (int64, m+1), idx (int32, nnz),
 * deg (int32, m); COO row and col (int32, nnz each).
 * gary_bin_info reports the format and sizes; the readers fill caller
 * buffers of those sizes (ptr: n+1 words, idx: nnz; src/dst: nnz each) and
 * check that the arrays agree; gary_bin_write_csr writes the CSR record,
 * deriving deg from ptr.  Errors: GARY_ERR_INPUT for unreadable, truncated or
 * inconsistent files. */
#define GARY_BIN_CSR 0u
#define GARY_BIN_COO 1u
int gary_bin_info(const char *path, uint32_t *format, uint32_t *n, uint64_t *nnz);
int gary_bin_read_csr(const char *path, uint64_t *ptr, uint32_t *idx);
int gary_bin_read_coo(const char *path, uint32_t *src, uint32_t *dst);
int gary_bin_write_csr(const char *path, const uint64_t *ptr, const uint32_t *idx, uint32_t n,
                       uint64_t nnz);

/* ---- seeded synthetic generators (host; RMAT also on the device) ------ *
 * Counter-based: edge i depends only on (seed, i), so any range can be
 * regenerated on the host to check a device batch. */
int gary_gen_er(uint32_t n, uint64_t m, uint64_t seed, uint32_t *src, uint32_t *dst);
int gary_gen_rmat(int scale, uint64_t seed, uint64_t first, uint64_t count, uint32_t *src,
                  uint32_t *dst);
int gary_gen_rmat_device(int scale, uint64_t seed, uint64_t first, uint64_t count,
                         uint32_t *d_src, uint32_t *d_dst, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* GARY_B200_H */
