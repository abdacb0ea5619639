// Batched set operations: the reference's include/ops layer as kernels.
//
//   gary_search_batch     binary_search (Search.cuh:48-61) and the two-phase
//                         cached search (Search.cuh:93-138) of many keys in one
//                         sorted list -- the kernels of test/SearchTest.cu:14-67
//   gary_intersect_batch  |A & B| (and A & B, sorted) for many pairs of sorted
//                         lists -- intersectBinarySearch (Intersection.cuh:18-135)
//                         and the merge / bitmap paths the reference stubs out
//                         (intersectMerge returns 0, Intersection.cuh:172-180)
//   gary_intersect_num_batch  the same counts restricted to members below a
//                         per-pair bound and outside a per-pair list of
//                         excluded ids -- the intersect_num family the
//                         reference leaves commented out (Intersection.cuh:361-485)
//
// Pair work is handed to warps by a persistent queue (32 pairs per grab).
// Variants:
//   MERGE   warp merge path: 32-wide windows of A and B, each lane locates its
//           A value in the B window with 5 shuffles, windows advance by ballots
//   SEARCH  lanes take the shorter list's values as keys and search the
//           longer list: phase 1 in 256 shared samples, phase 2 in HBM
//   BITMAP  the longer list as a shared-memory bitmap over 32K-value windows,
//           the shorter list probed window by window
//   AUTO    SEARCH when the longer list is much longer, else MERGE
// Materialised outputs are sorted (every variant emits in key order through
// ballot compaction); the reference's are unsorted (Intersection.cuh:24-47).
#include <cmath>
#include <vector>

#include "internal.cuh"
#include "pairs_gen.cuh"
#include "warp_ops.cuh"

namespace gary {
namespace {

constexpr int kSoWarps = 8;
constexpr uint32_t kSoWarpWords = 1024;  // per-warp shared words
constexpr uint32_t kSearchSamples = 256;
constexpr uint32_t kInf = 0xFFFFFFFFu;

struct PairView {
  const uint64_t *a_off, *b_off;
  const uint32_t *a_len, *b_len;
  const uint32_t *a, *b;
};

// Bounded / ancestor-filtered counts (the reference's intersect_num family,
// Intersection.cuh:361-485, left commented out there): per pair an exclusive
// upper bound on the members and a list of excluded ids.
struct PairFilter {
  const uint32_t *bound;   // per pair, or null
  const uint64_t *ex_off;  // per pair offsets into ex (npairs + 1), or null
  const uint32_t *ex;
};

// first index in [0, len) with l[i] >= x (all lanes compute the same answer)
__device__ __forceinline__ uint32_t so_lower_bound(const uint32_t *l, uint32_t len, uint32_t x) {
  uint32_t b = 0, e = len;
  while (b < e) {
    const uint32_t m = (b + e) >> 1;
    if (l[m] < x) b = m + 1;
    else e = m;
  }
  return b;
}

struct PairOut {
  uint64_t *counts;        // per pair, or null
  const uint64_t *out_off; // per pair, or null (count only)
  uint32_t *out;
};

__device__ __forceinline__ unsigned lanemask_lt(int lane) { return (1u << lane) - 1u; }

// ---- MERGE ------------------------------------------------------------------
__device__ uint32_t pair_merge(const uint32_t *A, uint32_t la, const uint32_t *B, uint32_t lb,
                               uint32_t *out, int lane) {
  uint32_t i = 0, j = 0, found_total = 0;
  while (i < la && j < lb) {
    const uint32_t av = i + lane < la ? A[i + lane] : kInf;
    const uint32_t bv = j + lane < lb ? B[j + lane] : kInf;
    const uint32_t a_last = __shfl_sync(kFull, av, min(31u, la - i - 1));
    const uint32_t b_last = __shfl_sync(kFull, bv, min(31u, lb - j - 1));
    // position of av in the B window: last k with B[k] <= av
    int lo = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
      const uint32_t v = __shfl_sync(kFull, bv, lo + step - 1);
      if (v <= av) lo += step;
    }
    const uint32_t cand = __shfl_sync(kFull, bv, lo);
    const uint32_t bprev = __shfl_sync(kFull, bv, lo > 0 ? lo - 1 : 0);
    const bool done_a = av != kInf && av <= b_last;
    const bool hit = done_a && (cand == av || (lo > 0 && bprev == av));
    const unsigned hm = __ballot_sync(kFull, hit);
    if (out && hit) out[found_total + __popc(hm & lanemask_lt(lane))] = av;
    found_total += __popc(hm);
    i += __popc(__ballot_sync(kFull, done_a));
    j += __popc(__ballot_sync(kFull, bv != kInf && bv <= a_last));
  }
  return found_total;
}

// ---- SEARCH (two-phase) ---------------------------------------------------
__device__ uint32_t pair_search(const uint32_t *S, uint32_t ls, const uint32_t *L, uint32_t ll,
                                uint32_t *cache, uint32_t *out, int lane) {
  const uint32_t ns = ll < kSearchSamples ? ll : kSearchSamples;
  for (uint32_t k = lane; k < ns; k += 32) cache[k] = L[(uint64_t)k * ll / ns];
  __syncwarp();
  uint32_t found_total = 0;
  for (uint32_t b = 0; b < ls; b += 32) {
    const bool ok = b + lane < ls;
    const uint32_t x = ok ? S[b + lane] : 0u;
    const bool hit = ok && search_2phase(L, ll, cache, ns, x);
    const unsigned hm = __ballot_sync(kFull, hit);
    if (out && hit) out[found_total + __popc(hm & lanemask_lt(lane))] = x;
    found_total += __popc(hm);
  }
  __syncwarp();
  return found_total;
}

// ---- BITMAP ---------------------------------------------------------------
// Windows of W = 32 * kSoWarpWords values.  In each non-empty window the
// warp sets the bits of L's values, probes S's values, then clears the words
// it set (so the bitmap starts every window zeroed).
__device__ uint32_t pair_bitmap(const uint32_t *S, uint32_t ls, const uint32_t *L, uint32_t ll,
                                uint32_t *bm, uint32_t *out, int lane) {
  constexpr uint32_t W = 32 * kSoWarpWords;
  uint32_t si = 0, li = 0, found_total = 0;
  while (si < ls && li < ll) {
    const uint32_t s0 = S[si], l0 = L[li];
    const uint32_t w0 = (s0 > l0 ? s0 : l0) / W * W;  // window holding the larger head
    const uint64_t w1 = (uint64_t)w0 + W;
    // skip values below the window
    auto lower = [&](const uint32_t *X, uint32_t n, uint32_t from, uint64_t v) {
      uint32_t b = from, e = n;  // first index with X[idx] >= v
      while (b < e) {
        const uint32_t mid = (b + e) >> 1;
        if (X[mid] < v) b = mid + 1;
        else e = mid;
      }
      return b;
    };
    const uint32_t sb = lower(S, ls, si, w0), se = lower(S, ls, sb, w1);
    const uint32_t lb = lower(L, ll, li, w0), le = lower(L, ll, lb, w1);
    for (uint32_t k = lb + lane; k < le; k += 32) {
      const uint32_t o = L[k] - w0;
      atomicOr(&bm[o >> 5], 1u << (o & 31));
    }
    __syncwarp();
    for (uint32_t k = sb; k < se; k += 32) {
      const bool ok = k + lane < se;
      const uint32_t x = ok ? S[k + lane] : w0;
      const uint32_t o = x - w0;
      const bool hit = ok && ((bm[o >> 5] >> (o & 31)) & 1u);
      const unsigned hm = __ballot_sync(kFull, hit);
      if (out && hit) out[found_total + __popc(hm & lanemask_lt(lane))] = x;
      found_total += __popc(hm);
    }
    __syncwarp();
    for (uint32_t k = lb + lane; k < le; k += 32) bm[(L[k] - w0) >> 5] = 0u;
    __syncwarp();
    si = se;
    li = le;
  }
  return found_total;
}

__global__ void __launch_bounds__(kSoWarps * 32)
    k_intersect_pairs(PairView pv, uint64_t npairs, int variant, PairOut po, PairFilter pf,
                      unsigned long long *queue, unsigned long long *total) {
  __shared__ __align__(16) uint32_t smem[kSoWarps * kSoWarpWords];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t *mine = smem + warp * kSoWarpWords;
  for (uint32_t i = lane; i < kSoWarpWords; i += 32) mine[i] = 0u;
  __syncwarp();
  unsigned long long local = 0;
  // One pair per claim: with Zipf lengths, claims of 32 pairs left warps
  // finishing their last long pairs while the rest idled (2^20 pairs at
  // overlap 0.1: AUTO 174 M pairs/s with 32 per claim, 214 M with 2, 235 M
  // with 1; one queue atomic per pair is far below what the L2 serves).
  while (true) {
    unsigned long long c = 0;
    if (lane == 0) c = atomicAdd(queue, 1ull);
    c = __shfl_sync(kFull, c, 0);
    if (c >= npairs) break;
    {
      const uint64_t p = c;
      uint32_t la = pv.a_len[p], lb = pv.b_len[p];
      const uint32_t *A = pv.a + pv.a_off[p], *B = pv.b + pv.b_off[p];
      const uint32_t bound = pf.bound ? pf.bound[p] : kInf;
      if (pf.bound) {  // members < bound only: both lists end at the bound
        la = so_lower_bound(A, la, bound);
        lb = so_lower_bound(B, lb, bound);
      }
      uint32_t *out = po.out_off ? po.out + po.out_off[p] : nullptr;
      uint32_t c2 = 0;
      if (la && lb) {
        // S: shorter (ties: A), L: longer
        const bool a_short = la <= lb;
        const uint32_t *S = a_short ? A : B, *L = a_short ? B : A;
        const uint32_t ls = a_short ? la : lb, ll = a_short ? lb : la;
        int v = variant;
        if (v == GARY_ISECT_AUTO) {
          // search once the longer list exceeds half of |S| log2 |L| (measured
          // on 2^20 Zipf pairs at overlap 0.1: 239 M pairs/s with the cut at
          // 4 |S| log2 |L|, 285 M at 1x, 301 M at 1/2, 290 M at 1/4)
          const uint32_t lg = 32 - __clz(ll);
          v = 2ull * ll > (uint64_t)ls * lg ? GARY_ISECT_SEARCH : GARY_ISECT_MERGE;
        }
        if (v == GARY_ISECT_MERGE) c2 = pair_merge(S, ls, L, ll, out, lane);
        else if (v == GARY_ISECT_SEARCH) c2 = pair_search(S, ls, L, ll, mine, out, lane);
        else {
          c2 = pair_bitmap(S, ls, L, ll, mine, out, lane);
        }
      }
      if (pf.ex_off && la && lb) {  // excluded ids that are members (each id once)
        const uint64_t e0 = pf.ex_off[p], e1 = pf.ex_off[p + 1];
        uint32_t drop = 0;
        for (uint64_t k = e0 + lane; k < e1; k += 32) {
          const uint32_t x = pf.ex[k];
          bool first = x < bound;
          for (uint64_t j = e0; first && j < k; ++j) first = pf.ex[j] != x;
          if (first) {
            const uint32_t ia = so_lower_bound(A, la, x), ib = so_lower_bound(B, lb, x);
            drop += ia < la && A[ia] == x && ib < lb && B[ib] == x;
          }
        }
        for (int o = 16; o; o >>= 1) drop += __shfl_xor_sync(kFull, drop, o);
        c2 -= drop;
      }
      if (lane == 0 && po.counts) po.counts[p] = c2;
      local += c2;
    }
  }
  if (lane == 0 && total && local) atomicAdd(total, local);
}

// ---- search batch ----------------------------------------------------------
__global__ void __launch_bounds__(256)
    k_search_batch(const uint32_t *__restrict__ list, uint64_t len, const uint32_t *__restrict__ keys,
                   uint64_t nkeys, uint32_t cache_n, uint8_t *__restrict__ found,
                   unsigned long long *count) {
  extern __shared__ uint32_t cache[];
  for (uint32_t k = threadIdx.x; k < cache_n; k += blockDim.x) cache[k] = list[(uint64_t)k * len / cache_n];
  __syncthreads();
  unsigned long long local = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nkeys;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t x = keys[i];
    uint32_t f;
    if (cache_n) {
      f = search_2phase(list, (uint32_t)len, cache, cache_n, x);
    } else {
      uint64_t b = 0, e = len;
      f = 0;
      while (b < e) {
        const uint64_t mid = (b + e) >> 1;
        const uint32_t v = list[mid];
        if (v == x) { f = 1; break; }
        if (v < x) b = mid + 1;
        else e = mid;
      }
    }
    if (found) found[i] = (uint8_t)f;
    local += f;
  }
  if (count) {
    local = warp_sum_u64(local);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(count, local);
  }
}

// ---- pair generation -------------------------------------------------------
__global__ void k_pair_lengths(PairGen pg, uint64_t first, uint64_t npairs, uint32_t *__restrict__ la,
                               uint32_t *__restrict__ lb, uint64_t *__restrict__ qa,
                               uint64_t *__restrict__ qb) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < npairs;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t a = pg.length(first + i, 0), b = pg.length(first + i, 1);
    la[i] = a;
    lb[i] = b;
    qa[i] = (a + 3) / 4;  // lists padded to 16 bytes
    qb[i] = (b + 3) / 4;
  }
}

__global__ void k_pair_values(PairGen pg, uint64_t first, uint64_t npairs,
                              const uint32_t *__restrict__ la, const uint32_t *__restrict__ lb,
                              const uint64_t *__restrict__ a_off, const uint64_t *__restrict__ b_off,
                              uint32_t *__restrict__ a, uint32_t *__restrict__ b) {
  const int lane = threadIdx.x & 31;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t i = warp; i < npairs; i += nwarps) {
    const uint32_t A = la[i], B = lb[i];
    const uint32_t pa = (A + 3) & ~3u, pb = (B + 3) & ~3u;
    for (uint32_t j = lane; j < pa; j += 32)
      a[a_off[i] + j] = j < A ? pg.value(first + i, 0, j, A, B) : kSentinel;
    for (uint32_t j = lane; j < pb; j += 32)
      b[b_off[i] + j] = j < B ? pg.value(first + i, 1, j, A, B) : kSentinel;
  }
}

PairGen make_gen(uint64_t seed, uint32_t nmax, const uint64_t *cdf, double overlap, uint64_t range) {
  PairGen g;
  g.key = pmix64(seed ^ 0x7F4A7C15F39CC060ull);
  g.range = range;
  const double t = overlap <= 0 ? 0.0 : (overlap >= 1 ? 4294967295.0 : overlap * 4294967296.0);
  g.overlap_thresh = (uint32_t)t;
  g.nmax = nmax;
  g.cdf = cdf;
  return g;
}

}  // namespace
}  // namespace gary

using namespace gary;

extern "C" int gary_zipf_table(uint32_t nmax, double s, uint64_t *cdf) {
  GARY_CHECK_ARG(nmax >= 1 && cdf, "need nmax >= 1 and an output table");
  GARY_CHECK_ARG(s > 0, "exponent must be positive");
  std::vector<long double> w(nmax);
  long double H = 0;
  for (uint32_t x = nmax; x >= 1; --x) {  // small terms first
    w[x - 1] = powl((long double)x, -(long double)s);
    H += w[x - 1];
  }
  long double c = 0;
  for (uint32_t k = 0; k + 1 < nmax; ++k) {
    c += w[k];
    long double f = c / H * 18446744073709551616.0L;
    cdf[k] = f >= 18446744073709551615.0L ? ~0ull : (uint64_t)f;
  }
  cdf[nmax - 1] = ~0ull;
  return GARY_OK;
}

extern "C" int gary_gen_pair_host(uint64_t seed, uint64_t pair, uint32_t nmax, const uint64_t *cdf,
                                  double overlap, uint64_t range, uint32_t *a, uint32_t *la,
                                  uint32_t *b, uint32_t *lb) {
  GARY_CHECK_ARG(cdf && la && lb, "NULL argument");
  GARY_CHECK_ARG(range >= (uint64_t)nmax && range <= (1ull << 32), "range must be in [nmax, 2^32]");
  const PairGen g = make_gen(seed, nmax, cdf, overlap, range);
  const uint32_t A = g.length(pair, 0), B = g.length(pair, 1);
  *la = A;
  *lb = B;
  if (a)
    for (uint32_t j = 0; j < A; ++j) a[j] = g.value(pair, 0, j, A, B);
  if (b)
    for (uint32_t j = 0; j < B; ++j) b[j] = g.value(pair, 1, j, A, B);
  return GARY_OK;
}

extern "C" int gary_gen_pairs_lengths(uint64_t seed, uint64_t first, uint64_t npairs, uint32_t nmax,
                                      const uint64_t *d_cdf, uint32_t *d_la, uint32_t *d_lb,
                                      uint64_t *d_qa, uint64_t *d_qb, void *stream) {
  GARY_CHECK_ARG(npairs == 0 || (d_cdf && d_la && d_lb && d_qa && d_qb), "NULL argument");
  if (!npairs) return GARY_OK;
  const PairGen g = make_gen(seed, nmax, d_cdf, 0.0, 1ull << 26);
  const uint64_t blocks = (npairs + 255) / 256, cap = (uint64_t)sm_count() * 16;
  k_pair_lengths<<<(unsigned)(blocks < cap ? blocks : cap), 256, 0, as_stream(stream)>>>(
      g, first, npairs, d_la, d_lb, d_qa, d_qb);
  GARY_CUDA(cudaGetLastError());
  return GARY_OK;
}

extern "C" int gary_gen_pairs_values(uint64_t seed, uint64_t first, uint64_t npairs, uint32_t nmax,
                                     const uint64_t *d_cdf, double overlap, uint64_t range,
                                     const uint32_t *d_la, const uint32_t *d_lb,
                                     const uint64_t *d_a_off, const uint64_t *d_b_off, uint32_t *d_a,
                                     uint32_t *d_b, void *stream) {
  GARY_CHECK_ARG(npairs == 0 || (d_cdf && d_la && d_lb && d_a_off && d_b_off && d_a && d_b),
                 "NULL argument");
  GARY_CHECK_ARG(range >= (uint64_t)nmax && range <= (1ull << 32), "range must be in [nmax, 2^32]");
  if (!npairs) return GARY_OK;
  const PairGen g = make_gen(seed, nmax, d_cdf, overlap, range);
  const uint64_t blocks = (npairs * 32 + 255) / 256, cap = (uint64_t)sm_count() * 16;
  k_pair_values<<<(unsigned)(blocks < cap ? blocks : cap), 256, 0, as_stream(stream)>>>(
      g, first, npairs, d_la, d_lb, d_a_off, d_b_off, d_a, d_b);
  GARY_CUDA(cudaGetLastError());
  return GARY_OK;
}

extern "C" int gary_intersect_batch(uint64_t npairs, const uint64_t *d_a_off, const uint32_t *d_a_len,
                                    const uint32_t *d_a, const uint64_t *d_b_off,
                                    const uint32_t *d_b_len, const uint32_t *d_b, int variant,
                                    uint64_t *d_counts, const uint64_t *d_out_off, uint32_t *d_out,
                                    uint64_t *d_total, uint64_t *d_queue, void *stream) {
  GARY_CHECK_ARG(variant >= GARY_ISECT_AUTO && variant <= GARY_ISECT_BITMAP, "unknown variant %d",
                 variant);
  GARY_CHECK_ARG(npairs == 0 || (d_a_off && d_a_len && d_a && d_b_off && d_b_len && d_b),
                 "NULL list argument");
  GARY_CHECK_ARG(!d_out_off || d_out, "d_out is NULL while d_out_off is set");
  GARY_CHECK_ARG(d_queue != nullptr, "d_queue (one device word of scheduler state) is NULL");
  cudaStream_t s = as_stream(stream);
  GARY_CUDA(cudaMemsetAsync(d_queue, 0, 8, s));
  if (d_total) GARY_CUDA(cudaMemsetAsync(d_total, 0, 8, s));
  if (!npairs) return GARY_OK;
  int per_sm = 0;
  GARY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_intersect_pairs, kSoWarps * 32, 0));
  if (per_sm < 1) per_sm = 1;
  const PairView pv{d_a_off, d_b_off, d_a_len, d_b_len, d_a, d_b};
  const PairOut po{d_counts, d_out_off, d_out};
  k_intersect_pairs<<<(unsigned)(sm_count() * per_sm), kSoWarps * 32, 0, s>>>(
      pv, npairs, variant, po, PairFilter{nullptr, nullptr, nullptr},
      reinterpret_cast<unsigned long long *>(d_queue), reinterpret_cast<unsigned long long *>(d_total));
  GARY_CUDA(cudaGetLastError());
  return GARY_OK;
}

extern "C" int gary_intersect_num_batch(uint64_t npairs, const uint64_t *d_a_off, const uint32_t *d_a_len,
                                        const uint32_t *d_a, const uint64_t *d_b_off,
                                        const uint32_t *d_b_len, const uint32_t *d_b, int variant,
                                        const uint32_t *d_bound, const uint64_t *d_ex_off,
                                        const uint32_t *d_ex, uint64_t *d_counts, uint64_t *d_total,
                                        uint64_t *d_queue, void *stream) {
  GARY_CHECK_ARG(variant >= GARY_ISECT_AUTO && variant <= GARY_ISECT_BITMAP, "unknown variant %d",
                 variant);
  GARY_CHECK_ARG(npairs == 0 || (d_a_off && d_a_len && d_a && d_b_off && d_b_len && d_b),
                 "NULL list argument");
  GARY_CHECK_ARG(!d_ex_off || d_ex, "d_ex is NULL while d_ex_off is set");
  GARY_CHECK_ARG(d_queue != nullptr, "d_queue (one device word of scheduler state) is NULL");
  cudaStream_t s = as_stream(stream);
  GARY_CUDA(cudaMemsetAsync(d_queue, 0, 8, s));
  if (d_total) GARY_CUDA(cudaMemsetAsync(d_total, 0, 8, s));
  if (!npairs) return GARY_OK;
  int per_sm = 0;
  GARY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_intersect_pairs, kSoWarps * 32, 0));
  if (per_sm < 1) per_sm = 1;
  const PairView pv{d_a_off, d_b_off, d_a_len, d_b_len, d_a, d_b};
  const PairOut po{d_counts, nullptr, nullptr};
  k_intersect_pairs<<<(unsigned)(sm_count() * per_sm), kSoWarps * 32, 0, s>>>(
      pv, npairs, variant, po, PairFilter{d_bound, d_ex_off, d_ex},
      reinterpret_cast<unsigned long long *>(d_queue), reinterpret_cast<unsigned long long *>(d_total));
  GARY_CUDA(cudaGetLastError());
  return GARY_OK;
}

extern "C" int gary_search_batch(const uint32_t *d_list, uint64_t len, const uint32_t *d_keys,
                                 uint64_t nkeys, uint32_t cache_entries, uint8_t *d_found,
                                 uint64_t *d_count, void *stream) {
  GARY_CHECK_ARG(len < (1ull << 32), "list longer than 2^32-1");
  GARY_CHECK_ARG(cache_entries <= 8192, "cache_entries must be <= 8192");
  GARY_CHECK_ARG(nkeys == 0 || (d_keys && (d_list || len == 0)), "NULL argument");
  cudaStream_t s = as_stream(stream);
  if (d_count) GARY_CUDA(cudaMemsetAsync(d_count, 0, 8, s));
  if (!nkeys) return GARY_OK;
  if (len == 0) {
    if (d_found) GARY_CUDA(cudaMemsetAsync(d_found, 0, nkeys, s));
    return GARY_OK;
  }
  const uint32_t cn = cache_entries && cache_entries > len ? (uint32_t)len : cache_entries;
  const uint64_t blocks = (nkeys + 255) / 256, cap = (uint64_t)sm_count() * 8;
  k_search_batch<<<(unsigned)(blocks < cap ? blocks : cap), 256, cn * 4, s>>>(
      d_list, len, d_keys, nkeys, cn, d_found, reinterpret_cast<unsigned long long *>(d_count));
  GARY_CUDA(cudaGetLastError());
  return GARY_OK;
}
