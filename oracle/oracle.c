/*
 * CPU oracle -- TEST INFRASTRUCTURE ONLY (see oracle.h).  Restates the
 * reference's counting-path algorithms in plain C; every function cites the
 * reference code it follows.  Nothing in the product links this file.
 */
#include "oracle.h"

#include <omp.h>
#include <stdlib.h>
#include <string.h>

/* ---- helpers ----------------------------------------------------------- */

/* LSD radix sort of 64-bit keys, 16-bit digits (4 passes). */
static void radix_sort_u64(uint64_t *a, int64_t n) {
  if (n < 2) return;
  uint64_t *tmp = (uint64_t *)malloc((size_t)n * sizeof(uint64_t));
  int64_t *cnt = (int64_t *)malloc(65536 * sizeof(int64_t));
  uint64_t *src = a, *dst = tmp;
  for (int pass = 0; pass < 4; ++pass) {
    const int sh = pass * 16;
    memset(cnt, 0, 65536 * sizeof(int64_t));
    for (int64_t i = 0; i < n; ++i) cnt[(src[i] >> sh) & 0xFFFF]++;
    int64_t s = 0;
    for (int d = 0; d < 65536; ++d) {
      int64_t c = cnt[d];
      cnt[d] = s;
      s += c;
    }
    for (int64_t i = 0; i < n; ++i) dst[cnt[(src[i] >> sh) & 0xFFFF]++] = src[i];
    uint64_t *t = src;
    src = dst;
    dst = t;
  }
  /* 4 passes: result is back in `a` */
  free(tmp);
  free(cnt);
}

static int64_t isect_count(const uint32_t *a, int64_t na, const uint32_t *b, int64_t nb) {
  int64_t i = 0, j = 0, c = 0;
  while (i < na && j < nb) {
    if (a[i] < b[j])
      ++i;
    else if (b[j] < a[i])
      ++j;
    else {
      ++c;
      ++i;
      ++j;
    }
  }
  return c;
}

static int before(uint32_t a, uint32_t b, const uint64_t *ptr) {
  uint64_t da = ptr[a + 1] - ptr[a], db = ptr[b + 1] - ptr[b];
  return da < db || (da == db && a < b);
}

/* ---- graph preparation ------------------------------------------------- */

/* GraphCOO::symmetrize (src/Graph.cpp:19-32) + toCSR_ (src/Graph.cpp:63-91),
 * plus the dedup and self-loop removal the synthetic configs require. */
int64_t orc_sym_csr(uint32_t n, int64_t m, const uint32_t *src, const uint32_t *dst,
                    uint64_t *ptr, uint32_t *idx) {
  uint64_t *keys = (uint64_t *)malloc((size_t)(2 * m + 1) * sizeof(uint64_t));
  int64_t k = 0;
  for (int64_t i = 0; i < m; ++i) {
    uint32_t a = src[i], b = dst[i];
    if (a == b || a >= n || b >= n) continue;
    keys[k++] = ((uint64_t)a << 32) | b;
    keys[k++] = ((uint64_t)b << 32) | a;
  }
  radix_sort_u64(keys, k);
  int64_t u = 0;
  for (int64_t i = 0; i < k; ++i)
    if (i == 0 || keys[i] != keys[i - 1]) keys[u++] = keys[i];
  memset(ptr, 0, ((size_t)n + 1) * sizeof(uint64_t));
  for (int64_t i = 0; i < u; ++i) {
    ptr[(keys[i] >> 32) + 1]++;
    idx[i] = (uint32_t)keys[i];
  }
  for (uint32_t v = 0; v < n; ++v) ptr[v + 1] += ptr[v];
  free(keys);
  return u;
}

/* GraphCOO::orientation (src/Graph.cpp:34-61) keeps src > dst; the degree
 * order keeps (deg u, u) < (deg v, v).  Lists stay sorted (filtering a sorted
 * list). */
void orc_orient(uint32_t n, const uint64_t *ptr, const uint32_t *idx, int by_degree,
                uint64_t *out_ptr, uint32_t *out_idx) {
  uint64_t k = 0;
  out_ptr[0] = 0;
  for (uint32_t v = 0; v < n; ++v) {
    for (uint64_t e = ptr[v]; e < ptr[v + 1]; ++e) {
      uint32_t w = idx[e];
      int keep = by_degree ? before(v, w, ptr) : (v > w);
      if (keep) out_idx[k++] = w;
    }
    out_ptr[v + 1] = k;
  }
}

/* ---- counting ---------------------------------------------------------- */

/* cpuTriCount (test/TriQueryTest.cu:17-37): for every v and u in N(v),
 * |N(u) & N(v)|, summed in uint64. */
uint64_t orc_tri_count(uint32_t n, const uint64_t *ptr, const uint32_t *idx, int threads) {
  uint64_t total = 0;
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : total)
  for (int64_t v = 0; v < (int64_t)n; ++v) {
    const uint32_t *av = idx + ptr[v];
    const int64_t dv = (int64_t)(ptr[v + 1] - ptr[v]);
    uint64_t local = 0;
    for (int64_t j = 0; j < dv; ++j) {
      const uint32_t u = av[j];
      local += (uint64_t)isect_count(idx + ptr[u], (int64_t)(ptr[u + 1] - ptr[u]), av, dv);
    }
    total += local;
  }
  return total;
}

uint64_t orc_k4_count(uint32_t n, const uint64_t *ptr, const uint32_t *idx, int threads) {
  uint64_t total = 0;
  uint32_t maxd = 0;
  for (uint32_t v = 0; v < n; ++v)
    if (ptr[v + 1] - ptr[v] > maxd) maxd = (uint32_t)(ptr[v + 1] - ptr[v]);
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel reduction(+ : total)
  {
    uint32_t *S = (uint32_t *)malloc(((size_t)maxd + 1) * sizeof(uint32_t));
#pragma omp for schedule(dynamic, 16)
    for (int64_t u = 0; u < (int64_t)n; ++u) {
      const uint32_t *au = idx + ptr[u];
      const int64_t du = (int64_t)(ptr[u + 1] - ptr[u]);
      for (int64_t j = 0; j < du; ++j) {
        const uint32_t v = au[j];
        const int64_t ns = orc_intersect(au, du, idx + ptr[v], (int64_t)(ptr[v + 1] - ptr[v]), S);
        for (int64_t t = 0; t < ns; ++t) {
          const uint32_t w = S[t];
          total += (uint64_t)isect_count(S, ns, idx + ptr[w], (int64_t)(ptr[w + 1] - ptr[w]));
        }
      }
    }
    free(S);
  }
  return total;
}

uint64_t orc_c4_count(uint32_t n, const uint64_t *ptr, const uint32_t *idx, int threads) {
  uint64_t total = 0;
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel reduction(+ : total)
  {
    uint32_t *cnt = (uint32_t *)calloc((size_t)n + 1, sizeof(uint32_t));
    uint32_t *touched = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
#pragma omp for schedule(dynamic, 64)
    for (int64_t uu = 0; uu < (int64_t)n; ++uu) {
      const uint32_t u = (uint32_t)uu;
      int64_t nt = 0;
      for (uint64_t e = ptr[u]; e < ptr[u + 1]; ++e) {
        const uint32_t v = idx[e];
        if (!before(v, u, ptr)) continue;
        for (uint64_t f = ptr[v]; f < ptr[v + 1]; ++f) {
          const uint32_t w = idx[f];
          if (!before(w, u, ptr)) continue;
          if (cnt[w]++ == 0) touched[nt++] = w;
        }
      }
      for (int64_t t = 0; t < nt; ++t) {
        const uint64_t c = cnt[touched[t]];
        total += c * (c - 1) / 2;
        cnt[touched[t]] = 0;
      }
    }
    free(cnt);
    free(touched);
  }
  return total;
}

uint64_t orc_c4_hom(uint32_t n, const uint64_t *ptr, const uint32_t *idx) {
  uint64_t total = 0;
  uint32_t *cnt = (uint32_t *)calloc((size_t)n + 1, sizeof(uint32_t));
  uint32_t *touched = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
  for (uint32_t u = 0; u < n; ++u) {
    int64_t nt = 0;
    for (uint64_t e = ptr[u]; e < ptr[u + 1]; ++e) {
      const uint32_t v = idx[e];
      for (uint64_t f = ptr[v]; f < ptr[v + 1]; ++f) {
        const uint32_t w = idx[f];
        if (cnt[w]++ == 0) touched[nt++] = w;
      }
    }
    for (int64_t t = 0; t < nt; ++t) {
      const uint64_t c = cnt[touched[t]];
      total += c * c;
      cnt[touched[t]] = 0;
    }
  }
  free(cnt);
  free(touched);
  return total;
}

void orc_tc_bytes(uint32_t n, const uint64_t *ptr, const uint32_t *idx, uint64_t *wedges,
                  uint64_t *alg_bytes) {
  uint64_t w = 0, b = 0;
  for (uint32_t u = 0; u < n; ++u) {
    const uint64_t du = ptr[u + 1] - ptr[u];
    for (uint64_t e = ptr[u]; e < ptr[u + 1]; ++e) {
      const uint32_t v = idx[e];
      const uint64_t dv = ptr[v + 1] - ptr[v];
      w += dv;
      b += 4 * (du + dv) + 24;
    }
  }
  *wedges = w;
  *alg_bytes = b;
}

/* ---- set operations ---------------------------------------------------- */

int64_t orc_intersect(const uint32_t *a, int64_t na, const uint32_t *b, int64_t nb,
                      uint32_t *out) {
  int64_t i = 0, j = 0, c = 0;
  while (i < na && j < nb) {
    if (a[i] < b[j])
      ++i;
    else if (b[j] < a[i])
      ++j;
    else {
      if (out) out[c] = a[i];
      ++c;
      ++i;
      ++j;
    }
  }
  return c;
}

/* Per-pair |A_i & B_i| of a pair batch by the same merge, OpenMP over pairs
 * (the reference's CPU check runs std::set_intersection one pair at a time,
 * test/SetOpTest.cu:94-95).  Returns the total. */
uint64_t orc_intersect_batch(int64_t npairs, const int64_t *a_off, const int32_t *la,
                             const uint32_t *a, const int64_t *b_off, const int32_t *lb,
                             const uint32_t *b, int64_t *counts, int threads) {
  uint64_t total = 0;
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : total)
  for (int64_t p = 0; p < npairs; ++p) {
    const int64_t c = orc_intersect(a + a_off[p], la[p], b + b_off[p], lb[p], NULL);
    if (counts) counts[p] = c;
    total += (uint64_t)c;
  }
  return total;
}

/* binary_search(span, key), include/ops/Search.cuh:48-61 */
int orc_binary_search(const uint32_t *list, int64_t n, uint32_t key) {
  int64_t l = 0, r = n - 1;
  while (r >= l) {
    int64_t mid = l + (r - l) / 2;
    uint32_t v = list[mid];
    if (v == key) return 1;
    if (v < key)
      l = mid + 1;
    else
      r = mid - 1;
  }
  return 0;
}

/* build_cache, include/ops/Search.cuh:93-100 */
void orc_build_cache(const uint32_t *list, int64_t n, int N, uint32_t *cache) {
  for (int i = 0; i < N; ++i) cache[i] = list[(int64_t)i * n / N];
}

/* binary_search_2phase, include/ops/Search.cuh:120-138: search the cache for
 * the last entry <= key (binary_search with pos, Search.cuh:67-81), then the
 * list range [pos*n/N, (pos+1)*n/N). */
int orc_binary_search_2phase(const uint32_t *list, int64_t n, const uint32_t *cache, int N,
                             uint32_t key) {
  int64_t l = 0, r = N - 1, pos = 0;
  while (r >= l) {
    pos = l + (r - l) / 2;
    uint32_t v = cache[pos];
    if (v == key) return 1;
    if (v < key)
      l = pos + 1;
    else
      r = pos - 1;
  }
  pos = r;
  if (pos < 0) return 0;
  int64_t bottom = pos * n / N, top = (pos + 1) * n / N;
  return orc_binary_search(list + bottom, top - bottom, key);
}

/* ---- cost-model network (FP64) ------------------------------------------ */
enum { NI = 6, NH1 = 64, NH2 = 64, NO = 4, OFF_W1 = 20, OFF_B1 = OFF_W1 + NH1 * NI,
       OFF_W2 = OFF_B1 + NH1, OFF_B2 = OFF_W2 + NH2 * NH1, OFF_W3 = OFF_B2 + NH2,
       OFF_B3 = OFF_W3 + NO * NH2, NPARAM = OFF_B3 + NO };

static void mlp_fwd1(const float *P, const float *x, double *h1, double *h2, double *y) {
  for (int i = 0; i < NH1; ++i) {
    double a = P[OFF_B1 + i];
    for (int f = 0; f < NI; ++f) a += (double)P[OFF_W1 + i * NI + f] * x[f];
    h1[i] = a > 0 ? a : 0;
  }
  for (int j = 0; j < NH2; ++j) {
    double a = P[OFF_B2 + j];
    for (int i = 0; i < NH1; ++i) a += (double)P[OFF_W2 + j * NH1 + i] * h1[i];
    h2[j] = a > 0 ? a : 0;
  }
  for (int k = 0; k < NO; ++k) {
    double a = P[OFF_B3 + k];
    for (int j = 0; j < NH2; ++j) a += (double)P[OFF_W3 + k * NH2 + j] * h2[j];
    y[k] = a;
  }
}

void orc_mlp_forward(const float *params, const float *x, int64_t n, double *y) {
  double h1[NH1], h2[NH2];
  for (int64_t s = 0; s < n; ++s) mlp_fwd1(params, x + s * NI, h1, h2, y + s * NO);
}

void orc_mlp_grad(const float *params, const float *x, const float *t, const uint8_t *mask,
                  int64_t n, double norm, double *grad, double *loss) {
  double h1[NH1], h2[NH2], y[NO], dy[NO], d2[NH2], d1[NH1];
  memset(grad, 0, NPARAM * sizeof(double));
  double L = 0;
  for (int64_t s = 0; s < n; ++s) {
    const float *xs = x + s * NI;
    mlp_fwd1(params, xs, h1, h2, y);
    for (int k = 0; k < NO; ++k) {
      const double e = ((mask[s] >> k) & 1) ? y[k] - t[s * NO + k] : 0.0;
      L += e * e;
      dy[k] = 2.0 * e / norm;
    }
    for (int j = 0; j < NH2; ++j) {
      double a = 0;
      for (int k = 0; k < NO; ++k) a += (double)params[OFF_W3 + k * NH2 + j] * dy[k];
      d2[j] = h2[j] > 0 ? a : 0;
    }
    for (int i = 0; i < NH1; ++i) {
      double a = 0;
      for (int j = 0; j < NH2; ++j) a += (double)params[OFF_W2 + j * NH1 + i] * d2[j];
      d1[i] = h1[i] > 0 ? a : 0;
    }
    for (int k = 0; k < NO; ++k) {
      for (int j = 0; j < NH2; ++j) grad[OFF_W3 + k * NH2 + j] += dy[k] * h2[j];
      grad[OFF_B3 + k] += dy[k];
    }
    for (int j = 0; j < NH2; ++j) {
      for (int i = 0; i < NH1; ++i) grad[OFF_W2 + j * NH1 + i] += d2[j] * h1[i];
      grad[OFF_B2 + j] += d2[j];
    }
    for (int i = 0; i < NH1; ++i) {
      for (int f = 0; f < NI; ++f) grad[OFF_W1 + i * NI + f] += d1[i] * xs[f];
      grad[OFF_B1 + i] += d1[i];
    }
  }
  *loss = L;
}

/* ---- the synthetic workload (see oracle.h) ------------------------------ */

static uint64_t orc_mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

void orc_gen_rmat(int scale, uint64_t seed, uint64_t first, uint64_t count, uint32_t *src,
                  uint32_t *dst) {
  const uint64_t golden = 0x9E3779B97F4A7C15ull;
  const uint32_t ta = (uint32_t)((57ull << 32) / 100), tb = (uint32_t)((76ull << 32) / 100),
                 tc = (uint32_t)((95ull << 32) / 100);
  const uint64_t key = orc_mix64(seed ^ 0x5851F42D4C957F2Dull);
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < (int64_t)count; ++k) {
    const uint64_t i = first + (uint64_t)k;
    uint32_t s = 0, d = 0;
    for (int l = 0; l < scale; l += 2) {
      const uint64_t r = orc_mix64(key + (i * 16 + (uint64_t)(l >> 1)) * golden);
      for (int h = 0; h < 2 && l + h < scale; ++h) {
        const uint32_t x = h ? (uint32_t)(r >> 32) : (uint32_t)r;
        s = (s << 1) | (uint32_t)(x >= tb);
        d = (d << 1) | (uint32_t)((x >= ta && x < tb) || x >= tc);
      }
    }
    src[k] = s;
    dst[k] = d;
  }
}

static int cmp_u32(const void *a, const void *b) {
  const uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
  return (x > y) - (x < y);
}

int64_t orc_unique_edges(uint32_t n, int64_t m, const uint32_t *src, const uint32_t *dst,
                         uint32_t *us, uint32_t *vs, int threads) {
  if (threads > 0) omp_set_num_threads(threads);
  uint64_t *off = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
  uint64_t *cur = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
  uint32_t *col = (uint32_t *)malloc((size_t)(m > 0 ? m : 1) * sizeof(uint32_t));
  uint64_t *keep = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
  /* rows by the smaller endpoint */
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m; ++i) {
    const uint32_t a = src[i], b = dst[i];
    if (a == b || a >= n || b >= n) continue;
    const uint32_t u = a < b ? a : b;
#pragma omp atomic
    off[u + 1]++;
  }
  for (uint32_t v = 0; v < n; ++v) off[v + 1] += off[v];
  memcpy(cur, off, ((size_t)n + 1) * sizeof(uint64_t));
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m; ++i) {
    const uint32_t a = src[i], b = dst[i];
    if (a == b || a >= n || b >= n) continue;
    const uint32_t u = a < b ? a : b, v = a < b ? b : a;
    uint64_t at;
#pragma omp atomic capture
    at = cur[u]++;
    col[at] = v;
  }
  /* sort and dedup every row in place; keep[u + 1] = its unique length */
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t u = 0; u < (int64_t)n; ++u) {
    uint32_t *r = col + off[u];
    const uint64_t len = off[u + 1] - off[u];
    if (len > 1) qsort(r, (size_t)len, sizeof(uint32_t), cmp_u32);
    uint64_t k = 0;
    for (uint64_t j = 0; j < len; ++j)
      if (j == 0 || r[j] != r[j - 1]) r[k++] = r[j];
    keep[u + 1] = k;
  }
  for (uint32_t v = 0; v < n; ++v) keep[v + 1] += keep[v];
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t u = 0; u < (int64_t)n; ++u) {
    const uint64_t k = keep[u + 1] - keep[u];
    for (uint64_t j = 0; j < k; ++j) {
      us[keep[u] + j] = (uint32_t)u;
      vs[keep[u] + j] = col[off[u] + j];
    }
  }
  const int64_t total = (int64_t)keep[n];
  free(off);
  free(cur);
  free(col);
  free(keep);
  return total;
}
