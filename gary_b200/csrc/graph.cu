// Graph construction on the device: symmetric CSR from an edge list, and the
// degree-oriented, relabeled, padded upload.  Replaces the reference's host
// pipeline (src/Graph.cpp:19-91 symmetrize / orientation / toCSR_, and
// src/DeviceGraph.cu:18-47 loadFromHost / populateDevice) with sort-based
// device passes: every step is a coalesced sweep or a CUB radix sort.
#include <cub/cub.cuh>
#include <thrust/execution_policy.h>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/reverse_iterator.h>
#include <thrust/iterator/transform_iterator.h>
#include <thrust/reduce.h>
#include <thrust/remove.h>
#include <thrust/scan.h>
#include <thrust/sequence.h>
#include <thrust/transform_reduce.h>
#include <thrust/unique.h>

#include <algorithm>
#include <exception>
#include <new>
#include <vector>

#include "graph.cuh"

struct gary_csr {
  int device = 0;
  uint32_t n = 0;
  uint64_t nnz = 0;
  gary::DevBuf<uint64_t> ptr;
  gary::DevBuf<uint32_t> idx;
};

namespace gary {
namespace {

constexpr int kThreads = 256;

inline unsigned grid_for(uint64_t items, int threads = kThreads) {
  uint64_t b = (items + threads - 1) / threads;
  uint64_t cap = (uint64_t)sm_count() * 16;
  if (b > cap) b = cap;
  return (unsigned)std::max<uint64_t>(b, 1);
}

inline int bits_for(uint64_t x) {  // bits needed to hold values in [0, x)
  int b = 0;
  while (b < 64 && (x - 1) >> b) ++b;
  return std::max(b, 1);
}

struct MaxU32 {
  __host__ __device__ uint32_t operator()(uint32_t a, uint32_t b) const { return a > b ? a : b; }
};
struct MinU64 {
  __host__ __device__ uint64_t operator()(uint64_t a, uint64_t b) const { return a < b ? a : b; }
};

// error bits written by validation kernels
enum : unsigned {
  kErrRange = 1u,
  kErrLoop = 2u,
  kErrOrder = 4u,
  kErrPtr = 8u,
  kErrDup = 16u,
  kErrAsym = 32u,
};

__global__ void k_degree(const uint64_t *__restrict__ ptr, uint32_t n, uint64_t nnz,
                         uint32_t *__restrict__ deg, unsigned *err) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t a = ptr[v], b = ptr[v + 1];
    if (b < a || b > nnz) {
      atomicOr(err, kErrPtr);
      deg[v] = 0;
    } else {
      deg[v] = (uint32_t)(b - a);
    }
  }
}

__global__ void k_indegree(const uint32_t *__restrict__ idx, uint64_t nnz, uint32_t n,
                           uint32_t *__restrict__ deg, unsigned *err) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < nnz;
       e += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t b = idx[e];
    if (b < n)
      atomicAdd(&deg[b], 1u);
    else
      atomicOr(err, kErrRange);
  }
}

__global__ void k_row_heads(const uint64_t *__restrict__ ptr, uint32_t n,
                            uint32_t *__restrict__ rowid) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t a = ptr[v];
    if (ptr[v + 1] > a) rowid[a] = (uint32_t)v;
  }
}

__global__ void k_rank_scatter(const uint32_t *__restrict__ perm, const uint32_t *__restrict__ deg,
                               uint32_t n, uint32_t *__restrict__ rank, uint32_t *__restrict__ rdeg) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    rank[perm[i]] = (uint32_t)i;
    rdeg[i] = deg[perm[i]];
  }
}

__device__ __forceinline__ bool before(uint32_t a, uint32_t b, const uint32_t *deg) {
  uint32_t da = deg[a], db = deg[b];
  return da < db || (da == db && a < b);
}

// One key per CSR entry: kept entries (a before b) become (rank a, rank b),
// the others ~0.  Symmetric input keeps exactly one copy of every edge.
// `dag` input keeps every entry, oriented.
__global__ void k_make_keys(const uint32_t *__restrict__ rowid, const uint32_t *__restrict__ idx,
                            uint64_t nnz, uint32_t n, const uint32_t *__restrict__ deg,
                            const uint32_t *__restrict__ rank, int lg, bool dag, bool validate,
                            uint64_t *__restrict__ keys, unsigned *err) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < nnz;
       e += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t a = rowid[e], b = idx[e];
    if (b >= n) {
      atomicOr(err, kErrRange);
      keys[e] = ~0ull;
      continue;
    }
    if (a == b) {
      atomicOr(err, kErrLoop);
      keys[e] = ~0ull;
      continue;
    }
    if (validate && e + 1 < nnz && rowid[e + 1] == a && idx[e + 1] <= b) atomicOr(err, kErrOrder);
    bool fwd = before(a, b, deg);
    if (!fwd && !dag) {
      keys[e] = ~0ull;
      continue;
    }
    uint32_t s = fwd ? a : b, t = fwd ? b : a;
    if (rank) {
      s = rank[s];
      t = rank[t];
    }
    keys[e] = ((uint64_t)s << lg) | t;
  }
}

// Ranked DAG without a global sort.  Pass 1 validates every CSR entry and
// counts the kept ones per ranked row (the row of the entry's earlier
// endpoint); pass 2 writes each kept entry's later endpoint into its row at
// an atomically claimed slot; a segmented sort then orders every row.
// Symmetric input keeps the copy stored in the earlier endpoint's row; `dag`
// input keeps every entry.
__device__ __forceinline__ bool kept_entry(uint32_t a, uint32_t b, const uint32_t *__restrict__ deg,
                                           bool dag, uint32_t &s, uint32_t &t) {
  const bool fwd = before(a, b, deg);
  if (!fwd && !dag) return false;
  s = fwd ? a : b;
  t = fwd ? b : a;
  return true;
}

// Per input entry e: its ranked row r = rank[s] and target rank[t], and its
// slot in row r (the old value of the row's count), so that the fill is a
// streaming pass.  Entries that are not kept get ent[e].x = kSentinel.
__global__ void k_count_rows(const uint32_t *__restrict__ rowid, const uint32_t *__restrict__ idx,
                             uint64_t nnz, uint32_t n, const uint32_t *__restrict__ deg,
                             const uint32_t *__restrict__ rank, bool dag, bool validate,
                             uint32_t *__restrict__ dplus, unsigned long long *__restrict__ kept,
                             unsigned *err, uint2 *__restrict__ ent, uint32_t *__restrict__ eslot) {
  unsigned long long mine = 0;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < nnz;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t a = rowid[e], b = idx[e];
    uint2 en = make_uint2(kSentinel, 0u);
    uint32_t slot = 0;
    uint32_t su, tv;
    if (b >= n) {
      atomicOr(err, kErrRange);
    } else if (a == b) {
      atomicOr(err, kErrLoop);
    } else {
      if (validate && e + 1 < nnz && rowid[e + 1] == a && idx[e + 1] <= b) atomicOr(err, kErrOrder);
      if (kept_entry(a, b, deg, dag, su, tv)) {
        en.x = rank[su];
        en.y = rank[tv];
        slot = atomicAdd(&dplus[en.x], 1u);
        ++mine;
      }
    }
    ent[e] = en;
    eslot[e] = slot;
  }
  for (int o = 16; o; o >>= 1) mine += __shfl_xor_sync(kFull, mine, o);
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd(kept, mine);
}

__global__ void k_fill_rows(const uint2 *__restrict__ ent, const uint32_t *__restrict__ eslot, uint64_t nnz,
                            const uint2 *__restrict__ row, uint32_t *__restrict__ adj) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < nnz;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint2 en = ent[e];
    if (en.x == kSentinel) continue;
    adj[(uint64_t)row[en.x].x * 4 + eslot[e]] = en.y;
  }
}

// plen4[u] = quads of u's padded list (whole octets)
__global__ void k_octet_quads(const uint32_t *__restrict__ dplus, uint32_t n, uint64_t *__restrict__ plen4) {
  for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n;
       u += (uint64_t)gridDim.x * blockDim.x)
    plen4[u] = ((dplus[u] + 7u) >> 3) << 1;
}

// A sorted row holding the same id twice: a duplicate edge in the input.
// Also wedge[u] = sum of d+(v) over v in N+(u); one warp per row.
__global__ void k_rows_check_wedges(const uint2 *__restrict__ row, const uint32_t *__restrict__ adj,
                                    uint32_t n, unsigned long long *__restrict__ wedge,
                                    unsigned *err) {
  const int lane = threadIdx.x & 31;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t u = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < n; u += warps) {
    const uint2 r = row[u];
    const uint32_t *l = adj + (uint64_t)r.x * 4;
    unsigned long long w = 0;
    bool dup = false;
    for (uint32_t k = lane; k < r.y; k += 32) {
      const uint32_t x = l[k];
      w += row[x].y;
      dup |= k + 1 < r.y && l[k + 1] == x;
    }
    for (int o = 16; o; o >>= 1) w += __shfl_xor_sync(kFull, w, o);
    if (__any_sync(kFull, dup) && lane == 0) atomicOr(err, kErrDup);
    if (lane == 0) wedge[u] = w;
  }
}

// ---- sorting the rows of a padded CSR in place ----------------------------
// Every row is sorted by a bitonic network held in registers:
// - up to 32 ids: one id per lane, several rows per warp in aligned segments
//   of 4, 8, 16 or 32 lanes (shuffles never leave a segment);
// - up to kSortWarpMax ids: one warp, E = 2..32 ids per lane;
// - up to kSortGroupMax ids: a group of 2, 4 or 8 warps with 32 ids per
//   lane, exchanging through shared memory only for strides of 1024 and up;
// - longer rows (rare): a library radix sort per row.
// Rows start 32-byte aligned and are padded with kSentinel to plen, a multiple
// of 8, so lanes load and store whole 8- or 16-byte vectors, positions from
// plen on are sentinels without a load, and sentinels sort last.
constexpr uint32_t kSortWarps = 8;
constexpr uint32_t kSortWarpMax = 1024;
constexpr uint32_t kSortGroupMax = 8192;
constexpr int kSortGroupThreads = 256;

__device__ __forceinline__ uint32_t keep_side(bool keep_min, uint32_t a, uint32_t b) {
  return keep_min ? min(a, b) : max(a, b);
}

// An S = 2^LOGS lane segment sorts one id per lane (sl = lane index in the segment).
template <int LOGS>
__device__ __forceinline__ uint32_t segment_sort(uint32_t x, int sl) {
#pragma unroll
  for (int lk = 1; lk <= LOGS; ++lk) {
#pragma unroll
    for (int lj = lk - 1; lj >= 0; --lj) {
      const uint32_t y = __shfl_xor_sync(kFull, x, 1 << lj);
      x = keep_side(((sl >> lj) & 1) == ((sl >> lk) & 1), x, y);
    }
  }
  return x;
}

// The rows of a warp's chunk (records in lane j's rec) whose length lies in
// (S/2, S] (from 2 for the smallest class): 32/S rows per pass, one segment each.
template <int LOGS>
__device__ __forceinline__ void sort_short_rows(uint2 rec, uint32_t *__restrict__ adj, int lane) {
  constexpr int S = 1 << LOGS;
  constexpr uint32_t lo = LOGS == 2 ? 2 : S / 2 + 1;
  uint32_t mask = __ballot_sync(kFull, rec.y >= lo && rec.y <= (uint32_t)S);
  const int seg = lane >> LOGS, sl = lane & (S - 1);
  while (mask) {
    const unsigned j = __fns(mask, 0, seg + 1);  // this segment's row, or none
    const int src = j < 32 ? (int)j : 0;
    const uint32_t rx = __shfl_sync(kFull, rec.x, src);
    const uint32_t dj = __shfl_sync(kFull, rec.y, src);
    const uint32_t d = j < 32 ? dj : 0u;
    uint32_t *l = adj + (uint64_t)rx * 4;
    uint32_t x = (uint32_t)sl < d ? l[sl] : kSentinel;
    x = segment_sort<LOGS>(x, sl);
    if ((uint32_t)sl < d) l[sl] = x;
    const unsigned cut = __fns(mask, 0, 32 / S + 1);  // first row of the next pass
    mask = cut < 32 ? mask & ~((1u << cut) - 1) : 0u;
  }
}

// One warp's block of a bitonic network, E = 2^LOGE ids per lane: lane L
// owns elements gbase .. gbase+E-1 of the row (gbase = its offset in the
// row).  Strides below E compare two registers of one lane; strides below
// 32E pair a register with the same register of lane L ^ (j/E).  The
// direction of each comparison follows bit k of the element's index.
template <int LOGE>
__device__ __forceinline__ void warp_stage(uint32_t (&x)[1 << LOGE], int lane, uint32_t gbase, uint32_t k,
                                           int lj) {
  constexpr int E = 1 << LOGE;
  if (lj >= LOGE) {
    const int lm = 1 << (lj - LOGE);
    const bool keep_min = ((lane & lm) == 0) == ((gbase & k) == 0);
#pragma unroll
    for (int e = 0; e < E; ++e) x[e] = keep_side(keep_min, x[e], __shfl_xor_sync(kFull, x[e], lm));
  } else {
    const uint32_t j = 1u << lj;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      if (e & j) continue;
      const int f = e | j;
      const bool up = k < (uint32_t)E ? (e & k) == 0 : (gbase & k) == 0;
      const uint32_t lo = min(x[e], x[f]), hi = max(x[e], x[f]);
      x[e] = up ? lo : hi;
      x[f] = up ? hi : lo;
    }
  }
}

// All stages of the network whose sequence length k is at most 32E: sorts
// the warp's block, ascending or descending by bit 32E of gbase.
template <int LOGE>
__device__ __forceinline__ void warp_sort_block(uint32_t (&x)[1 << LOGE], int lane, uint32_t gbase) {
#pragma unroll
  for (int lk = 1; lk <= LOGE + 5; ++lk)
#pragma unroll
    for (int lj = lk - 1; lj >= 0; --lj) warp_stage<LOGE>(x, lane, gbase, 1u << lk, lj);
}

// The strides below 32E of a merge of sequence length k > 32E.
template <int LOGE>
__device__ __forceinline__ void warp_merge_block(uint32_t (&x)[1 << LOGE], int lane, uint32_t gbase, uint32_t k) {
#pragma unroll
  for (int lj = LOGE + 4; lj >= 0; --lj) warp_stage<LOGE>(x, lane, gbase, k, lj);
}

// Sorts one padded row of up to 2^(LOGE+5+LOGW) ids with a group of 2^LOGW
// warps (wg = warp index in the group): lane L of warp wg owns elements from
// gbase = (wg*32 + L)*E.  Strides of 32E and up pair a register with the same
// register of warp wg ^ (j/32E), through xs (layout [warp][e][lane]) and a
// named barrier per group.
template <int LOGE, int LOGW>
__device__ __forceinline__ void group_sort_row(uint32_t *__restrict__ l, uint32_t plen, int lane, int wg,
                                               uint32_t *xs, int bar_id) {
  constexpr int E = 1 << LOGE;
  constexpr int LOGWARP = LOGE + 5;
  const uint32_t gbase = ((uint32_t)wg * 32 + lane) * E;
  uint32_t x[E];
  if constexpr (E == 2) {
    uint2 v = make_uint2(kSentinel, kSentinel);
    if (gbase < plen) v = *reinterpret_cast<const uint2 *>(l + gbase);
    x[0] = v.x;
    x[1] = v.y;
  } else {
#pragma unroll
    for (int q = 0; q < E / 4; ++q) {
      uint4 v = make_uint4(kSentinel, kSentinel, kSentinel, kSentinel);
      if (gbase + 4 * q < plen) v = *reinterpret_cast<const uint4 *>(l + gbase + 4 * q);
      x[4 * q] = v.x;
      x[4 * q + 1] = v.y;
      x[4 * q + 2] = v.z;
      x[4 * q + 3] = v.w;
    }
  }
  warp_sort_block<LOGE>(x, lane, gbase);
  if constexpr (LOGW > 0) {
#pragma unroll 1
    for (int lk = LOGWARP + 1; lk <= LOGWARP + LOGW; ++lk) {
      const uint32_t k = 1u << lk;
#pragma unroll 1
      for (int lj = lk - 1; lj >= LOGWARP; --lj) {
        const int wm = 1 << (lj - LOGWARP);
        const bool keep_min = ((wg & wm) == 0) == ((gbase & k) == 0);
#pragma unroll
        for (int e = 0; e < E; ++e) xs[(wg * E + e) * 32 + lane] = x[e];
        asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(32 << LOGW) : "memory");
#pragma unroll
        for (int e = 0; e < E; ++e) x[e] = keep_side(keep_min, x[e], xs[((wg ^ wm) * E + e) * 32 + lane]);
        asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(32 << LOGW) : "memory");
      }
      warp_merge_block<LOGE>(x, lane, gbase, k);
    }
  }
  if constexpr (E == 2) {
    if (gbase < plen) *reinterpret_cast<uint2 *>(l + gbase) = make_uint2(x[0], x[1]);
  } else {
#pragma unroll
    for (int q = 0; q < E / 4; ++q)
      if (gbase + 4 * q < plen)
        *reinterpret_cast<uint4 *>(l + gbase + 4 * q) = make_uint4(x[4 * q], x[4 * q + 1], x[4 * q + 2], x[4 * q + 3]);
  }
}

__device__ __forceinline__ uint32_t padded_len(uint32_t d) { return ((d + 7) >> 3) << 3; }

// A warp takes 32 consecutive rows (one coalesced load of their records):
// the short ones by segments, then the others up to kSortWarpMax one by one.
__global__ void __launch_bounds__(kSortWarps * 32)
    k_sort_rows_warp(const uint2 *__restrict__ row, uint32_t n, uint32_t *__restrict__ adj) {
  const int lane = threadIdx.x & 31;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t c = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; c * 32 < n; c += warps) {
    const uint64_t u0 = c * 32;
    const uint2 rec = u0 + lane < n ? row[u0 + lane] : make_uint2(0, 0);
    sort_short_rows<2>(rec, adj, lane);
    sort_short_rows<3>(rec, adj, lane);
    sort_short_rows<4>(rec, adj, lane);
    sort_short_rows<5>(rec, adj, lane);
    uint32_t mask = __ballot_sync(kFull, rec.y > 32 && rec.y <= kSortWarpMax);
    while (mask) {
      const int j = __ffs(mask) - 1;
      mask &= mask - 1;
      const uint32_t rx = __shfl_sync(kFull, rec.x, j), d = __shfl_sync(kFull, rec.y, j);
      uint32_t *l = adj + (uint64_t)rx * 4;
      const uint32_t plen = padded_len(d);
      if (d <= 64) group_sort_row<1, 0>(l, plen, lane, 0, nullptr, 0);
      else if (d <= 128) group_sort_row<2, 0>(l, plen, lane, 0, nullptr, 0);
      else if (d <= 256) group_sort_row<3, 0>(l, plen, lane, 0, nullptr, 0);
      else if (d <= 512) group_sort_row<4, 0>(l, plen, lane, 0, nullptr, 0);
      else group_sort_row<5, 0>(l, plen, lane, 0, nullptr, 0);
    }
  }
}

// Rows longer than kSortWarpMax, sorted into lists by length class:
// (1024, 2048], (2048, 4096], (4096, 8192] and longer.
__global__ void k_long_rows(const uint2 *__restrict__ row, uint32_t n, uint32_t cap,
                            uint32_t *__restrict__ lists, uint32_t *__restrict__ counts) {
  for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n;
       u += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t d = row[u].y;
    if (d <= kSortWarpMax) continue;
    const int cls = d <= 2048 ? 0 : d <= 4096 ? 1 : d <= kSortGroupMax ? 2 : 3;
    const uint32_t slot = atomicAdd(&counts[cls], 1u);
    if (slot < cap) lists[(uint64_t)cls * cap + slot] = (uint32_t)u;
  }
}

// Rows of the length class of 2^LOGW warps per group; kSortGroupThreads /
// (32 << LOGW) groups per CTA, each on its own rows and named barrier.
template <int LOGW>
__global__ void __launch_bounds__(kSortGroupThreads)
    k_sort_rows_group(const uint2 *__restrict__ row, const uint32_t *__restrict__ list,
                      const uint32_t *__restrict__ count, uint32_t cap, uint32_t *__restrict__ adj) {
  constexpr int G = kSortGroupThreads / (32 << LOGW);
  __shared__ uint32_t xs[kSortGroupThreads * 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = warp >> LOGW, wg = warp & ((1 << LOGW) - 1);
  uint32_t *gx = xs + (uint32_t)g * (1024u << LOGW);
  const uint32_t nl = min(*count, cap);
  for (uint32_t t = blockIdx.x * G + g; t < nl; t += gridDim.x * G) {
    const uint2 r = row[list[t]];
    group_sort_row<5, LOGW>(adj + (uint64_t)r.x * 4, padded_len(r.y), lane, wg, gx, 1 + g);
  }
}

struct RowOf {
  const uint2 *row;
  __host__ __device__ uint2 operator()(uint32_t u) const { return row[u]; }
};


__global__ void k_check_unique(const uint64_t *__restrict__ keys, uint64_t m, unsigned *err) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i + 1 < m;
       i += (uint64_t)gridDim.x * blockDim.x)
    if (keys[i] == keys[i + 1]) atomicOr(err, kErrDup);
}

// rowstart[u] = index of the first key of row u (or of the next row); keys sorted.
__global__ void k_key_heads(const uint64_t *__restrict__ keys, uint64_t m, int lg,
                            uint64_t *__restrict__ rowstart) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t u = keys[i] >> lg;
    if (i == 0 || (keys[i - 1] >> lg) != u) rowstart[u] = i;
  }
}

__global__ void k_rows(const uint64_t *__restrict__ rowstart, uint32_t n,
                       uint32_t *__restrict__ dplus, uint64_t *__restrict__ plen4) {
  for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n;
       u += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t d = (uint32_t)(rowstart[u + 1] - rowstart[u]);
    dplus[u] = d;
    plen4[u] = ((d + 7u) >> 3) << 1;  // whole octets: 32-byte aligned, padded to 8 words
  }
}

__global__ void k_scatter_adj(const uint64_t *__restrict__ keys, uint64_t m, int lg,
                              const uint64_t *__restrict__ rowstart,
                              const uint64_t *__restrict__ off4, uint32_t *__restrict__ adj) {
  const uint64_t mask = (1ull << lg) - 1;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t k = keys[i];
    uint64_t u = k >> lg;
    adj[off4[u] * 4 + (i - rowstart[u])] = (uint32_t)(k & mask);
  }
}

__global__ void k_row_records(const uint64_t *__restrict__ off4, const uint32_t *__restrict__ dplus,
                              uint32_t n, uint2 *__restrict__ row, uint64_t *__restrict__ indptr) {
  for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u <= n;
       u += (uint64_t)gridDim.x * blockDim.x) {
    indptr[u] = off4[u] * 4;
    if (u < n) row[u] = make_uint2((uint32_t)off4[u], dplus[u]);
  }
}

// wedge[u] = sum of d+(v) over v in N+(u).  Keys are sorted, so equal rows
// are contiguous lanes: a segmented warp scan leaves each run's sum in its
// last lane, which issues one atomic per run.
__global__ void k_wedges(const uint64_t *__restrict__ keys, uint64_t m, int lg,
                         const uint32_t *__restrict__ dplus, unsigned long long *__restrict__ wedge) {
  const uint64_t mask = (1ull << lg) - 1;
  const int lane = threadIdx.x & 31;
  uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x; base < m; base += stride) {
    uint64_t i = base + threadIdx.x;
    bool ok = i < m;
    uint64_t k = ok ? keys[i] : ~0ull;
    uint32_t u = ok ? (uint32_t)(k >> lg) : 0xFFFFFFFFu;
    unsigned long long v = ok ? dplus[k & mask] : 0ull;
    for (int o = 1; o < 32; o <<= 1) {
      unsigned long long t = __shfl_up_sync(kFull, v, o);
      uint32_t tu = __shfl_up_sync(kFull, u, o);
      if (lane >= o && tu == u) v += t;
    }
    uint32_t nu = __shfl_down_sync(kFull, u, 1);
    bool tail = lane == 31 || nu != u;
    if (ok && tail && v) atomicAdd(&wedge[u], v);
  }
}

struct Sq {
  __host__ __device__ uint64_t operator()(uint32_t d) const { return (uint64_t)d * d; }
};

// ---- CUB helpers with stream-ordered temporaries ------------------------
int radix_sort_keys(DevBuf<uint64_t> &keys, DevBuf<uint64_t> &alt, uint64_t m, int end_bit,
                    cudaStream_t s) {
  cub::DoubleBuffer<uint64_t> db(keys.p, alt.p);
  size_t tmp = 0;
  GARY_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp, db, m, 0, end_bit, s));
  DevBuf<uint8_t> t;
  GARY_TRY(t.alloc(tmp, s));
  GARY_CUDA(cub::DeviceRadixSort::SortKeys(t.p, tmp, db, m, 0, end_bit, s));
  if (db.Current() != keys.p) std::swap(keys, alt);
  return GARY_OK;
}

int row_starts(const DevBuf<uint64_t> &keys, uint64_t m, uint32_t n, int lg,
               DevBuf<uint64_t> &rowstart, cudaStream_t s, bool persistent = false) {
  if (persistent) GARY_TRY(rowstart.alloc_persistent((uint64_t)n + 1));
  else GARY_TRY(rowstart.alloc((uint64_t)n + 1, s));
  // fill with m, heads, then reverse min-scan so empty rows point at the next row
  ScratchAlloc pol_alloc{s};
  auto pol = thrust::cuda::par_nosync(pol_alloc).on(s);
  thrust::fill(pol, rowstart.p, rowstart.p + n + 1, m);
  if (m) k_key_heads<<<grid_for(m), kThreads, 0, s>>>(keys.p, m, lg, rowstart.p);
  auto rb = thrust::make_reverse_iterator(rowstart.p + n + 1);
  thrust::inclusive_scan(pol, rb, rb + n + 1, rb, MinU64());
  GARY_CUDA(cudaGetLastError());
  return GARY_OK;
}

int read_err(unsigned *d_err, cudaStream_t s, unsigned *h) {
  GARY_CUDA(cudaMemcpyAsync(h, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  GARY_CUDA(cudaStreamSynchronize(s));
  return GARY_OK;
}

int input_error(unsigned bits) {
  set_error("malformed graph input:%s%s%s%s%s%s", (bits & kErrRange) ? " id>=n" : "",
            (bits & kErrLoop) ? " self-loop" : "", (bits & kErrOrder) ? " unsorted-list" : "",
            (bits & kErrPtr) ? " bad-ptr" : "", (bits & kErrDup) ? " duplicate-edge" : "",
            (bits & kErrAsym) ? " not-symmetric" : "");
  return GARY_ERR_INPUT;
}

}  // namespace

// ---------------------------------------------------------------------------
// Stream compaction with 64-bit sizes (CUB DeviceSelect takes int64 counts;
// arrays here exceed 2^31 entries for graphs of ~10^9 edges).
namespace {
struct NotAllOnes {
  __host__ __device__ bool operator()(uint64_t k) const { return k != ~0ull; }
};
}  // namespace

int compact_keys(DevBuf<uint64_t> &keys, uint64_t count, uint64_t &kept, cudaStream_t s) {
  kept = 0;
  if (!count) return GARY_OK;
  DevBuf<uint64_t> out, nsel;
  GARY_TRY(out.alloc(count, s));
  GARY_TRY(nsel.alloc(1, s));
  size_t tmp = 0;
  GARY_CUDA(cub::DeviceSelect::If(nullptr, tmp, keys.p, out.p, nsel.p, (int64_t)count, NotAllOnes(), s));
  DevBuf<uint8_t> t;
  GARY_TRY(t.alloc(tmp, s));
  GARY_CUDA(cub::DeviceSelect::If(t.p, tmp, keys.p, out.p, nsel.p, (int64_t)count, NotAllOnes(), s));
  GARY_CUDA(cudaMemcpyAsync(&kept, nsel.p, 8, cudaMemcpyDeviceToHost, s));
  GARY_CUDA(cudaStreamSynchronize(s));
  std::swap(keys, out);
  return GARY_OK;
}

int unique_keys(DevBuf<uint64_t> &keys, uint64_t count, uint64_t &kept, cudaStream_t s) {
  kept = 0;
  if (!count) return GARY_OK;
  DevBuf<uint64_t> out, nsel;
  GARY_TRY(out.alloc(count, s));
  GARY_TRY(nsel.alloc(1, s));
  size_t tmp = 0;
  GARY_CUDA(cub::DeviceSelect::Unique(nullptr, tmp, keys.p, out.p, nsel.p, (int64_t)count, s));
  DevBuf<uint8_t> t;
  GARY_TRY(t.alloc(tmp, s));
  GARY_CUDA(cub::DeviceSelect::Unique(t.p, tmp, keys.p, out.p, nsel.p, (int64_t)count, s));
  GARY_CUDA(cudaMemcpyAsync(&kept, nsel.p, 8, cudaMemcpyDeviceToHost, s));
  GARY_CUDA(cudaStreamSynchronize(s));
  std::swap(keys, out);
  return GARY_OK;
}

// ---------------------------------------------------------------------------
// Padded lists from sorted (row << lg | col) keys.
int padded_from_keys(const DevBuf<uint64_t> &keys, uint64_t m, uint32_t n, int lg, PaddedCSR &c,
                     cudaStream_t s) {
  ScratchAlloc pol_alloc{s};
  auto pol = thrust::cuda::par_nosync(pol_alloc).on(s);
  c.n = n;
  c.m = m;
  DevBuf<uint64_t> rowstart, off4;
  GARY_TRY(row_starts(keys, m, n, lg, rowstart, s));
  GARY_TRY(c.outdeg.alloc_persistent(n));
  GARY_TRY(off4.alloc((uint64_t)n + 1, s));
  k_rows<<<grid_for(n), kThreads, 0, s>>>(rowstart.p, n, c.outdeg.p, off4.p);
  thrust::exclusive_scan(pol, off4.p, off4.p + n + 1, off4.p, 0ull);
  uint64_t quads = 0;
  GARY_CUDA(cudaMemcpyAsync(&quads, off4.p + n, 8, cudaMemcpyDeviceToHost, s));
  GARY_CUDA(cudaStreamSynchronize(s));
  if (quads >= (1ull << 32)) {
    set_error("graph too large: %llu padded words", (unsigned long long)quads * 4);
    return GARY_ERR_UNSUPPORTED;
  }
  c.words = quads * 4;
  // 4 slack words: 32-byte-aligned octet reads of the last list stay in bounds
  GARY_TRY(c.adj.alloc_persistent(c.words + 4));
  GARY_CUDA(cudaMemsetAsync(c.adj.p, 0xFF, c.adj.bytes(), s));
  if (m) k_scatter_adj<<<grid_for(m), kThreads, 0, s>>>(keys.p, m, lg, rowstart.p, off4.p, c.adj.p);
  GARY_TRY(c.row.alloc_persistent(n));
  GARY_TRY(c.indptr.alloc_persistent((uint64_t)n + 1));
  k_row_records<<<grid_for((uint64_t)n + 1), kThreads, 0, s>>>(off4.p, c.outdeg.p, n, c.row.p,
                                                              c.indptr.p);
  GARY_CUDA(cudaGetLastError());
  c.max_len = thrust::reduce(pol, c.outdeg.p, c.outdeg.p + n, 0u, MaxU32());
  return GARY_OK;
}

// The ranked DAG's padded lists straight from the CSR entries (count, fill,
// segmented sort; no sort of all edges), plus per-vertex wedge counts.
int ranked_dag_by_rows(const uint32_t *rowid, const uint32_t *didx, uint64_t nnz, uint32_t n,
                       const uint32_t *deg, const uint32_t *rank, bool dag, bool validate,
                       unsigned *err, PaddedCSR &c, DevBuf<uint64_t> &wedge, uint64_t &m,
                       cudaStream_t s) {
  ScratchAlloc pol_alloc{s};
  auto pol = thrust::cuda::par_nosync(pol_alloc).on(s);
  PhaseTrace tr("dag rows", s);
  c.n = n;
  GARY_TRY(c.outdeg.alloc_persistent(n));
  GARY_CUDA(cudaMemsetAsync(c.outdeg.p, 0, (uint64_t)n * 4, s));
  DevBuf<unsigned long long> dkept;
  GARY_TRY(dkept.alloc(1, s));
  GARY_CUDA(cudaMemsetAsync(dkept.p, 0, 8, s));
  DevBuf<uint2> ent;      // per entry: ranked row, target rank
  DevBuf<uint32_t> eslot; // per entry: slot in its row
  GARY_TRY(ent.alloc(std::max<uint64_t>(nnz, 1), s));
  GARY_TRY(eslot.alloc(std::max<uint64_t>(nnz, 1), s));
  if (nnz)
    k_count_rows<<<grid_for(nnz), kThreads, 0, s>>>(rowid, didx, nnz, n, deg, rank, dag, validate,
                                                    c.outdeg.p, dkept.p, err, ent.p, eslot.p);
  GARY_CUDA(cudaGetLastError());
  DevBuf<uint64_t> off4;
  GARY_TRY(off4.alloc((uint64_t)n + 1, s));
  k_octet_quads<<<grid_for(n), kThreads, 0, s>>>(c.outdeg.p, n, off4.p);
  GARY_CUDA(cudaMemsetAsync(off4.p + n, 0, 8, s));
  thrust::exclusive_scan(pol, off4.p, off4.p + n + 1, off4.p, 0ull);
  uint64_t quads = 0;
  unsigned long long km = 0;
  unsigned herr = 0;
  tr.mark("count");
  GARY_CUDA(cudaMemcpyAsync(&quads, off4.p + n, 8, cudaMemcpyDeviceToHost, s));
  GARY_CUDA(cudaMemcpyAsync(&km, dkept.p, 8, cudaMemcpyDeviceToHost, s));
  GARY_TRY(read_err(err, s, &herr));
  if (herr) return input_error(herr);
  m = km;
  c.m = m;
  if (!dag && 2 * m != nnz) return input_error(kErrAsym);
  if (quads >= (1ull << 32)) {
    set_error("graph too large: %llu padded words", (unsigned long long)quads * 4);
    return GARY_ERR_UNSUPPORTED;
  }
  c.words = quads * 4;
  GARY_TRY(c.adj.alloc_persistent(c.words + 4));
  GARY_CUDA(cudaMemsetAsync(c.adj.p, 0xFF, c.adj.bytes(), s));
  GARY_TRY(c.row.alloc_persistent(n));
  GARY_TRY(c.indptr.alloc_persistent((uint64_t)n + 1));
  k_row_records<<<grid_for((uint64_t)n + 1), kThreads, 0, s>>>(off4.p, c.outdeg.p, n, c.row.p,
                                                              c.indptr.p);
  GARY_CUDA(cudaGetLastError());
  off4.release();
  tr.mark("allocate + records");
  if (nnz) k_fill_rows<<<grid_for(nnz), kThreads, 0, s>>>(ent.p, eslot.p, nnz, c.row.p, c.adj.p);
  GARY_CUDA(cudaGetLastError());
  ent.release();
  eslot.release();
  tr.mark("fill");
  // order every row in place
  if (m) {
    int per_sm = 0;
    GARY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sort_rows_warp, kSortWarps * 32, 0));
    k_sort_rows_warp<<<sm_count() * std::max(per_sm, 1), kSortWarps * 32, 0, s>>>(c.row.p, n, c.adj.p);
    GARY_CUDA(cudaGetLastError());
    tr.mark("row sort: up to 1024 ids (warp)");
    // at most m / 1025 rows are longer than 1024 ids
    const uint32_t cap = (uint32_t)std::min<uint64_t>(n, m / (kSortWarpMax + 1) + 1);
    DevBuf<uint32_t> lists, counts;
    GARY_TRY(lists.alloc((uint64_t)cap * 4, s));
    GARY_TRY(counts.alloc(4, s));
    GARY_CUDA(cudaMemsetAsync(counts.p, 0, 16, s));
    k_long_rows<<<grid_for(n), kThreads, 0, s>>>(c.row.p, n, cap, lists.p, counts.p);
    GARY_CUDA(cudaGetLastError());
    auto group_launch = [&](auto kern, int cls) -> int {
      int b = 0;
      GARY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, kSortGroupThreads, 0));
      kern<<<sm_count() * std::max(b, 1), kSortGroupThreads, 0, s>>>(c.row.p, lists.p + (uint64_t)cls * cap,
                                                                      counts.p + cls, cap, c.adj.p);
      GARY_CUDA(cudaGetLastError());
      return GARY_OK;
    };
    GARY_TRY(group_launch(k_sort_rows_group<1>, 0));
    GARY_TRY(group_launch(k_sort_rows_group<2>, 1));
    GARY_TRY(group_launch(k_sort_rows_group<3>, 2));
    tr.mark("row sort: up to 8192 ids (warp groups)");
    uint32_t nh = 0;
    GARY_CUDA(cudaMemcpyAsync(&nh, counts.p + 3, 4, cudaMemcpyDeviceToHost, s));
    GARY_CUDA(cudaStreamSynchronize(s));
    if (nh) {  // the longest rows (rare; d+ above 8192): one library radix sort per row
      std::vector<uint2> hr(nh);
      DevBuf<uint2> rr;
      GARY_TRY(rr.alloc(nh, s));
      const uint32_t *l3 = lists.p + 3ull * cap;
      thrust::transform(pol, l3, l3 + nh, rr.p, RowOf{c.row.p});
      GARY_CUDA(cudaMemcpyAsync(hr.data(), rr.p, (uint64_t)nh * 8, cudaMemcpyDeviceToHost, s));
      GARY_CUDA(cudaStreamSynchronize(s));
      uint32_t dmax = 0;
      for (const uint2 &r : hr) dmax = std::max(dmax, r.y);
      DevBuf<uint32_t> tmpk;
      GARY_TRY(tmpk.alloc(dmax, s));
      size_t tmp = 0;
      GARY_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp, c.adj.p, tmpk.p, (int)dmax, 0, 32, s));
      DevBuf<uint8_t> t;
      GARY_TRY(t.alloc(std::max<size_t>(tmp, 1), s));
      for (const uint2 &r : hr) {
        uint32_t *l = c.adj.p + (uint64_t)r.x * 4;
        size_t tb = tmp;
        GARY_CUDA(cub::DeviceRadixSort::SortKeys(t.p, tb, l, tmpk.p, (int)r.y, 0, 32, s));
        GARY_CUDA(cudaMemcpyAsync(l, tmpk.p, (uint64_t)r.y * 4, cudaMemcpyDeviceToDevice, s));
      }
    }
  }
  tr.mark("row sort: longer rows");
  GARY_TRY(wedge.alloc_persistent(n));
  k_rows_check_wedges<<<grid_for((uint64_t)n * 32), kThreads, 0, s>>>(
      c.row.p, c.adj.p, n, reinterpret_cast<unsigned long long *>(wedge.p), err);
  GARY_CUDA(cudaGetLastError());
  if (validate || dag) {
    GARY_TRY(read_err(err, s, &herr));
    if (herr) return input_error(herr);
  }
  c.max_len = thrust::reduce(pol, c.outdeg.p, c.outdeg.p + n, 0u, MaxU32());
  return GARY_OK;
}

// Oriented keys of every CSR entry, compacted and sorted.  rank == nullptr:
// caller ids; else degree ranks.
int oriented_keys(const uint32_t *rowid, const uint32_t *didx, uint64_t nnz, uint32_t n,
                  const uint32_t *deg, const uint32_t *rank, int lg, bool dag, bool validate,
                  unsigned *err, DevBuf<uint64_t> &keys, uint64_t &m, cudaStream_t s) {
  ScratchAlloc pol_alloc{s};
  auto pol = thrust::cuda::par_nosync(pol_alloc).on(s);
  m = 0;
  GARY_TRY(keys.alloc(std::max<uint64_t>(nnz, 1), s));
  if (nnz) {
    k_make_keys<<<grid_for(nnz), kThreads, 0, s>>>(rowid, didx, nnz, n, deg, rank, lg, dag,
                                                   validate, keys.p, err);
    GARY_CUDA(cudaGetLastError());
    GARY_TRY(compact_keys(keys, nnz, m, s));
  }
  DevBuf<uint64_t> alt;
  GARY_TRY(alt.alloc(std::max<uint64_t>(m, 1), s));
  if (m) GARY_TRY(radix_sort_keys(keys, alt, m, 2 * lg, s));
  return GARY_OK;
}

// ---------------------------------------------------------------------------
// Oriented upload.  Input CSR (symmetric or DAG) -> degree-oriented padded lists.
namespace {
// group id of caller vertex v: the g with off[g] <= v < off[g + 1]
__global__ void k_group_ids(const uint64_t *__restrict__ off, uint32_t ngroups, uint32_t n,
                            uint32_t *__restrict__ gid) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t b = 0, e = ngroups;  // last g with off[g] <= v
    while (e - b > 1) {
      const uint32_t m = (b + e) >> 1;
      if (off[m] <= v) b = m;
      else e = m;
    }
    gid[v] = b;
  }
}
__global__ void k_rank_keys(const uint32_t *__restrict__ deg, const uint32_t *__restrict__ gid,
                            uint32_t n, int degbits, uint64_t *__restrict__ key) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x)
    key[v] = ((gid ? (uint64_t)gid[v] : 0ull) << degbits) | deg[v];
}
__global__ void k_gather_u32(const uint32_t *__restrict__ perm, const uint32_t *__restrict__ src,
                             uint32_t n, uint32_t *__restrict__ dst) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    dst[i] = src[perm[i]];
}
}  // namespace

// group_off (host, ngroups + 1 entries; may be null): vertices
// [group_off[g], group_off[g+1]) form graph g of a disjoint union.  Ranks are
// then taken within each graph, so every graph keeps a contiguous rank range.
// Host ids copied in chunks on a side stream, so that the upload's stream can
// run what needs only the offsets while they cross PCIe.  wait(k) makes the
// upload's stream wait for chunk k; the destructor makes it wait for every
// chunk, so a stream-ordered free of the destination on that stream (error
// paths included) never overtakes a copy.
struct ChunkedCopy {
  static constexpr int kMaxChunks = 8;
  cudaStream_t s = nullptr, side = nullptr;
  cudaEvent_t done[kMaxChunks] = {};
  uint64_t off[kMaxChunks + 1] = {};
  int chunks = 0;
  ChunkedCopy() = default;
  ChunkedCopy(const ChunkedCopy &) = delete;
  ChunkedCopy &operator=(const ChunkedCopy &) = delete;
  int start(uint32_t *dst, const uint32_t *src, uint64_t count, cudaStream_t stream) {
    s = stream;
    GARY_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    cudaEvent_t ready;
    GARY_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
    cudaEventRecord(ready, s);  // dst was allocated on s
    cudaStreamWaitEvent(side, ready, 0);
    cudaEventDestroy(ready);
    const uint64_t min_chunk = 1ull << 24;  // ids
    chunks = (int)std::min<uint64_t>(kMaxChunks, std::max<uint64_t>(1, count / min_chunk));
    for (int k = 0; k <= chunks; ++k) off[k] = count * (uint64_t)k / (uint64_t)chunks;
    for (int k = 0; k < chunks; ++k) {
      GARY_CUDA(cudaEventCreateWithFlags(&done[k], cudaEventDisableTiming));
      GARY_CUDA(cudaMemcpyAsync(dst + off[k], src + off[k], (off[k + 1] - off[k]) * 4,
                                cudaMemcpyHostToDevice, side));
      GARY_CUDA(cudaEventRecord(done[k], side));
    }
    return GARY_OK;
  }
  void wait(int k) const {
    if (k < chunks && done[k]) cudaStreamWaitEvent(s, done[k], 0);
  }
  ~ChunkedCopy() {
    for (int k = 0; k < chunks; ++k)
      if (done[k]) {
        cudaStreamWaitEvent(s, done[k], 0);
        cudaEventDestroy(done[k]);
      }
    if (side) cudaStreamDestroy(side);
  }
};

int upload(const uint64_t *ptr, const uint32_t *idx, uint32_t n, uint64_t nnz, uint32_t flags,
           cudaStream_t s, gary_graph **out, const uint64_t *group_off, uint32_t ngroups) {
  const bool on_dev = flags & GARY_INPUT_DEVICE;
  const bool dag = flags & GARY_INPUT_DAG;
  const bool keep_ids = flags & GARY_KEEP_IDS;
  const bool validate = flags & GARY_VALIDATE;
  GARY_CHECK_ARG(out != nullptr, "out is NULL");
  GARY_CHECK_ARG(n > 0 && n < 0xFFFFFFFFu, "n must be in [1, 2^32-1)");
  GARY_CHECK_ARG(ptr != nullptr, "ptr is NULL");
  GARY_CHECK_ARG(nnz == 0 || idx != nullptr, "idx is NULL");
  if (!on_dev) {
    GARY_CHECK_ARG(ptr[0] == 0 && ptr[n] == nnz, "ptr[0] must be 0 and ptr[n] must equal nnz");
  }
  *out = nullptr;

  auto g = std::make_unique<gary_graph>();
  GARY_CUDA(cudaGetDevice(&g->device));
  g->n = n;
  g->flags = flags;
  g->keep_ids = keep_ids;
  ScratchAlloc pol_alloc{s};
  auto pol = thrust::cuda::par_nosync(pol_alloc).on(s);
  PhaseTrace tr("upload", s);

  // 1. input on the device.  From host memory the offsets come first on s and
  // the ids in chunks on a side stream; s meanwhile derives what needs only
  // the offsets (degrees of symmetric input, row ids, and for symmetric input
  // the ranks too) and, for DAG input, counts in-degrees chunk by chunk.
  DevBuf<uint64_t> dptr_own;
  DevBuf<uint32_t> didx_own;
  const uint64_t *dptr = ptr;
  const uint32_t *didx = idx;
  ChunkedCopy ids;  // after didx_own: destroyed first, so s waits for the copies before the free
  if (!on_dev) {
    GARY_TRY(dptr_own.alloc((uint64_t)n + 1, s));
    GARY_TRY(didx_own.alloc(nnz, s));
    GARY_CUDA(cudaMemcpyAsync(dptr_own.p, ptr, ((uint64_t)n + 1) * 8, cudaMemcpyHostToDevice, s));
    if (nnz) GARY_TRY(ids.start(didx_own.p, idx, nnz, s));
    dptr = dptr_own.p;
    didx = didx_own.p;
  }
  auto wait_ids = [&] {
    for (int k = 0; k < ids.chunks; ++k) ids.wait(k);
  };

  DevBuf<unsigned> err;
  GARY_TRY(err.alloc(1, s));
  GARY_CUDA(cudaMemsetAsync(err.p, 0, sizeof(unsigned), s));

  // 2. degrees (undirected)
  DevBuf<uint32_t> deg;
  GARY_TRY(deg.alloc(n, s));
  k_degree<<<grid_for(n), kThreads, 0, s>>>(dptr, n, nnz, deg.p, err.p);
  // row id of every entry: heads, then an inclusive max-scan (offsets only)
  const int lg = bits_for(n);
  DevBuf<uint32_t> rowid;
  GARY_TRY(rowid.alloc(nnz, s));
  if (nnz) {
    GARY_CUDA(cudaMemsetAsync(rowid.p, 0, nnz * 4, s));
    k_row_heads<<<grid_for(n), kThreads, 0, s>>>(dptr, n, rowid.p);
    size_t tmp = 0;
    GARY_CUDA(cub::DeviceScan::InclusiveScan(nullptr, tmp, rowid.p, rowid.p, MaxU32(), nnz, s));
    DevBuf<uint8_t> t;
    GARY_TRY(t.alloc(tmp, s));
    GARY_CUDA(cub::DeviceScan::InclusiveScan(t.p, tmp, rowid.p, rowid.p, MaxU32(), nnz, s));
  }
  if (dag && nnz) {
    if (ids.chunks) {
      for (int k = 0; k < ids.chunks; ++k) {
        ids.wait(k);
        const uint64_t len = ids.off[k + 1] - ids.off[k];
        k_indegree<<<grid_for(len), kThreads, 0, s>>>(didx + ids.off[k], len, n, deg.p, err.p);
      }
    } else {
      k_indegree<<<grid_for(nnz), kThreads, 0, s>>>(didx, nnz, n, deg.p, err.p);
    }
  }
  GARY_CUDA(cudaGetLastError());
  if (on_dev) {
    uint64_t ends[2];
    GARY_CUDA(cudaMemcpyAsync(&ends[0], dptr, 8, cudaMemcpyDeviceToHost, s));
    GARY_CUDA(cudaMemcpyAsync(&ends[1], dptr + n, 8, cudaMemcpyDeviceToHost, s));
    GARY_CUDA(cudaStreamSynchronize(s));
    GARY_CHECK_ARG(ends[0] == 0 && ends[1] == nnz, "ptr[0] must be 0 and ptr[n] must equal nnz");
  }
  g->max_degree = thrust::reduce(pol, deg.p, deg.p + n, 0u, MaxU32());

  tr.mark("h2d offsets, degrees, row ids");
  // 3. ranks by (graph, degree, id): a stable radix sort of the ids
  DevBuf<uint32_t> rank, gidc;
  if (ngroups) {
    GARY_CHECK_ARG(group_off[0] == 0 && group_off[ngroups] == n,
                   "group offsets must start at 0 and end at n");
    for (uint32_t k = 0; k < ngroups; ++k)
      GARY_CHECK_ARG(group_off[k] <= group_off[k + 1], "group offsets must be non-decreasing");
    g->group_off.assign(group_off, group_off + ngroups + 1);
    DevBuf<uint64_t> doff;
    GARY_TRY(doff.alloc((uint64_t)ngroups + 1, s));
    GARY_CUDA(cudaMemcpyAsync(doff.p, group_off, ((uint64_t)ngroups + 1) * 8, cudaMemcpyHostToDevice, s));
    GARY_TRY(gidc.alloc(n, s));
    k_group_ids<<<grid_for(n), kThreads, 0, s>>>(doff.p, ngroups, n, gidc.p);
    GARY_CUDA(cudaGetLastError());
  }
  {
    const int degbits = bits_for((uint64_t)g->max_degree + 1);
    const int keybits = degbits + (ngroups ? bits_for(ngroups) : 0);
    DevBuf<uint64_t> dk, dk2;
    DevBuf<uint32_t> perm2;
    GARY_TRY(dk.alloc(n, s));
    GARY_TRY(dk2.alloc(n, s));
    GARY_TRY(g->perm.alloc_persistent(n));
    GARY_TRY(perm2.alloc(n, s));  // scratch: releasing a persistent block synchronises the device
    k_rank_keys<<<grid_for(n), kThreads, 0, s>>>(deg.p, ngroups ? gidc.p : nullptr, n, degbits, dk.p);
    thrust::sequence(pol, perm2.p, perm2.p + n, 0u);
    cub::DoubleBuffer<uint64_t> kb(dk.p, dk2.p);
    cub::DoubleBuffer<uint32_t> vb(perm2.p, g->perm.p);
    size_t tmp = 0;
    GARY_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, kb, vb, n, 0, keybits, s));
    DevBuf<uint8_t> t;
    GARY_TRY(t.alloc(tmp, s));
    GARY_CUDA(cub::DeviceRadixSort::SortPairs(t.p, tmp, kb, vb, n, 0, keybits, s));
    if (vb.Current() != g->perm.p)
      GARY_CUDA(cudaMemcpyAsync(g->perm.p, vb.Current(), (uint64_t)n * 4, cudaMemcpyDeviceToDevice, s));
    GARY_TRY(rank.alloc(n, s));
    GARY_TRY(g->rdeg.alloc_persistent(n));
    k_rank_scatter<<<grid_for(n), kThreads, 0, s>>>(g->perm.p, deg.p, n, rank.p, g->rdeg.p);
    if (ngroups) {
      g->ngroups = ngroups;
      GARY_TRY(g->gid.alloc_persistent(n));
      k_gather_u32<<<grid_for(n), kThreads, 0, s>>>(g->perm.p, gidc.p, n, g->gid.p);
    }
    GARY_CUDA(cudaGetLastError());
  }

  tr.mark("ranks");
  // 4. the ids themselves from here on
  wait_ids();
  tr.mark("h2d ids (rest)");
  // 5. the ranked DAG's padded lists, validated; per-vertex wedge counts
  uint64_t m = 0;
  GARY_TRY(ranked_dag_by_rows(rowid.p, didx, nnz, n, deg.p, rank.p, dag, validate, err.p, g->dag,
                              g->wedge, m, s));
  tr.mark("rows: count, fill, sort");
  // 6. statistics
  g->out_deg_sq = thrust::transform_reduce(pol, g->dag.outdeg.p, g->dag.outdeg.p + n, Sq(), 0ull,
                                           thrust::plus<uint64_t>());
  g->wedges = thrust::reduce(pol, g->wedge.p, g->wedge.p + n, 0ull);
  g->alg_bytes = 4 * g->out_deg_sq + 4 * g->wedges + 24 * m;
  tr.mark("statistics");

  // 7. the same orientation in caller ids, for the views (GARY_KEEP_IDS)
  if (keep_ids) {
    DevBuf<uint64_t> keys;
    uint64_t m2 = 0;
    GARY_TRY(oriented_keys(rowid.p, didx, nnz, n, deg.p, nullptr, lg, dag, false, err.p, keys, m2, s));
    GARY_TRY(padded_from_keys(keys, m2, n, lg, g->kept, s));
  }
  GARY_CUDA(cudaEventCreate(&g->ev0));
  GARY_CUDA(cudaEventCreate(&g->ev1));
  GARY_CUDA(cudaStreamSynchronize(s));
  *out = g.release();
  return GARY_OK;
}

// ---------------------------------------------------------------------------
// Symmetric CSR from an undirected edge list (dedup, drop loops, symmetrise).
namespace {
__global__ void k_edge_keys(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst,
                            uint64_t m, uint32_t n, int lg, uint64_t *__restrict__ keys,
                            unsigned *err) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t a = src[i], b = dst[i];
    if (a >= n || b >= n) {
      atomicOr(err, kErrRange);
      keys[2 * i] = keys[2 * i + 1] = ~0ull;
    } else if (a == b) {
      keys[2 * i] = keys[2 * i + 1] = ~0ull;
    } else {
      keys[2 * i] = ((uint64_t)a << lg) | b;
      keys[2 * i + 1] = ((uint64_t)b << lg) | a;
    }
  }
}
__global__ void k_key_cols(const uint64_t *__restrict__ keys, uint64_t m, int lg,
                           uint32_t *__restrict__ idx) {
  const uint64_t mask = (1ull << lg) - 1;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m;
       i += (uint64_t)gridDim.x * blockDim.x)
    idx[i] = (uint32_t)(keys[i] & mask);
}
}  // namespace

int csr_from_edges(const uint32_t *src, const uint32_t *dst, uint64_t m, uint32_t n,
                   uint32_t flags, cudaStream_t s, gary_csr **out) {
  GARY_CHECK_ARG(out != nullptr, "out is NULL");
  GARY_CHECK_ARG(n > 0 && n < 0xFFFFFFFFu, "n must be in [1, 2^32-1)");
  GARY_CHECK_ARG(m == 0 || (src && dst), "src/dst is NULL");
  *out = nullptr;
  auto c = std::make_unique<gary_csr>();
  GARY_CUDA(cudaGetDevice(&c->device));
  c->n = n;
  ScratchAlloc pol_alloc{s};
  auto pol = thrust::cuda::par_nosync(pol_alloc).on(s);
  const int lg = bits_for(n);
  DevBuf<uint32_t> s_own, d_own;
  if (!(flags & GARY_INPUT_DEVICE) && m) {
    GARY_TRY(s_own.alloc(m, s));
    GARY_TRY(d_own.alloc(m, s));
    GARY_CUDA(cudaMemcpyAsync(s_own.p, src, m * 4, cudaMemcpyHostToDevice, s));
    GARY_CUDA(cudaMemcpyAsync(d_own.p, dst, m * 4, cudaMemcpyHostToDevice, s));
    src = s_own.p;
    dst = d_own.p;
  }
  DevBuf<unsigned> err;
  GARY_TRY(err.alloc(1, s));
  GARY_CUDA(cudaMemsetAsync(err.p, 0, 4, s));
  DevBuf<uint64_t> keys, alt;
  uint64_t k = 0;
  GARY_TRY(keys.alloc(std::max<uint64_t>(2 * m, 1), s));
  if (m) {
    k_edge_keys<<<grid_for(m), kThreads, 0, s>>>(src, dst, m, n, lg, keys.p, err.p);
    GARY_CUDA(cudaGetLastError());
    GARY_TRY(compact_keys(keys, 2 * m, k, s));
  }
  s_own.release();
  d_own.release();
  unsigned herr = 0;
  GARY_TRY(read_err(err.p, s, &herr));
  if (herr) return input_error(herr);
  GARY_TRY(alt.alloc(std::max<uint64_t>(k, 1), s));
  if (k) {
    GARY_TRY(radix_sort_keys(keys, alt, k, 2 * lg, s));
    GARY_TRY(unique_keys(keys, k, k, s));
  }
  alt.release();
  DevBuf<uint64_t> rowstart;
  GARY_TRY(row_starts(keys, k, n, lg, rowstart, s, true));
  GARY_TRY(c->idx.alloc_persistent(std::max<uint64_t>(k, 1)));
  if (k) k_key_cols<<<grid_for(k), kThreads, 0, s>>>(keys.p, k, lg, c->idx.p);
  GARY_CUDA(cudaGetLastError());
  c->ptr = std::move(rowstart);
  c->nnz = k;
  GARY_CUDA(cudaStreamSynchronize(s));
  *out = c.release();
  return GARY_OK;
}

// ---------------------------------------------------------------------------
// Unpadded host copies and the COO view.
namespace {
// heads for the padded layout: rowid of every padded word (kSentinel padding
// words are dropped afterwards)
__global__ void k_padded_heads(const uint2 *__restrict__ row, uint32_t n,
                               uint32_t *__restrict__ rowid) {
  for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n;
       u += (uint64_t)gridDim.x * blockDim.x) {
    uint2 r = row[u];
    if (r.y) rowid[(uint64_t)r.x * 4] = (uint32_t)u;
  }
}
struct IsReal {
  const uint32_t *adj;
  __host__ __device__ bool operator()(uint64_t w) const { return adj[w] != kSentinel; }
};
__global__ void k_gather_pairs(const uint64_t *__restrict__ words, uint64_t m,
                               const uint32_t *__restrict__ rowid, const uint32_t *__restrict__ adj,
                               uint32_t *__restrict__ r, uint32_t *__restrict__ c) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t w = words[i];
    r[i] = rowid[w];
    c[i] = adj[w];
  }
}
}  // namespace

int padded_rowid(const PaddedCSR &c, DevBuf<uint32_t> &rowid, cudaStream_t s) {
  GARY_TRY(rowid.alloc(std::max<uint64_t>(c.words, 1), s));
  if (!c.words) return GARY_OK;
  GARY_CUDA(cudaMemsetAsync(rowid.p, 0, c.words * 4, s));
  k_padded_heads<<<grid_for(c.n), kThreads, 0, s>>>(c.row.p, c.n, rowid.p);
  size_t tmp = 0;
  GARY_CUDA(cub::DeviceScan::InclusiveScan(nullptr, tmp, rowid.p, rowid.p, MaxU32(), c.words, s));
  DevBuf<uint8_t> t;
  GARY_TRY(t.alloc(tmp, s));
  GARY_CUDA(cub::DeviceScan::InclusiveScan(t.p, tmp, rowid.p, rowid.p, MaxU32(), c.words, s));
  return GARY_OK;
}

int build_coo(PaddedCSR &c, cudaStream_t s) {
  if (c.coo_row.p || c.m == 0) return GARY_OK;
  ScratchAlloc pol_alloc{s};
  auto pol = thrust::cuda::par_nosync(pol_alloc).on(s);
  DevBuf<uint32_t> rowid;
  GARY_TRY(padded_rowid(c, rowid, s));
  DevBuf<uint64_t> words, nsel;
  GARY_TRY(words.alloc(c.m, s));
  GARY_TRY(nsel.alloc(1, s));
  uint64_t got = 0;
  {
    cub::CountingInputIterator<uint64_t> it(0);
    size_t tmp = 0;
    GARY_CUDA(cub::DeviceSelect::If(nullptr, tmp, it, words.p, nsel.p, (int64_t)c.words, IsReal{c.adj.p}, s));
    DevBuf<uint8_t> t;
    GARY_TRY(t.alloc(tmp, s));
    GARY_CUDA(cub::DeviceSelect::If(t.p, tmp, it, words.p, nsel.p, (int64_t)c.words, IsReal{c.adj.p}, s));
    GARY_CUDA(cudaMemcpyAsync(&got, nsel.p, 8, cudaMemcpyDeviceToHost, s));
    GARY_CUDA(cudaStreamSynchronize(s));
  }
  if (got != c.m) {
    set_error("internal: padded adjacency holds %llu ids, expected %llu",
              (unsigned long long)got, (unsigned long long)c.m);
    return GARY_ERR_CUDA;
  }
  GARY_TRY(c.coo_row.alloc_persistent(c.m));
  GARY_TRY(c.coo_col.alloc_persistent(c.m));
  k_gather_pairs<<<grid_for(c.m), kThreads, 0, s>>>(words.p, c.m, rowid.p, c.adj.p, c.coo_row.p,
                                                    c.coo_col.p);
  GARY_CUDA(cudaGetLastError());
  GARY_CUDA(cudaStreamSynchronize(s));
  return GARY_OK;
}

namespace {
// both directions of every oriented edge, from the padded DAG
__global__ void k_sym_keys(const uint2 *__restrict__ row, const uint32_t *__restrict__ adj,
                           const uint32_t *__restrict__ rowid, uint64_t words, int lg,
                           uint64_t *__restrict__ keys) {
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < words;
       w += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t u = rowid[w];
    const uint2 r = row[u];
    const uint64_t pos = w - (uint64_t)r.x * 4;
    if (pos < r.y) {
      const uint64_t v = adj[w];
      keys[2 * w] = ((uint64_t)u << lg) | v;
      keys[2 * w + 1] = (v << lg) | u;
    } else {
      keys[2 * w] = keys[2 * w + 1] = ~0ull;
    }
  }
}
}  // namespace

// Symmetric lists in rank ids (for 4-cycle counting), built once on demand.
int build_symmetric(gary_graph *g, cudaStream_t s) {
  if (g->sym.row.p) return GARY_OK;
  ScratchAlloc pol_alloc{s};
  auto pol = thrust::cuda::par_nosync(pol_alloc).on(s);
  const uint32_t n = g->n;
  const int lg = bits_for(n);
  const uint64_t W = g->dag.words;
  DevBuf<uint64_t> keys;
  uint64_t m2 = 0;
  {
    DevBuf<uint32_t> rowid;
    GARY_TRY(padded_rowid(g->dag, rowid, s));
    GARY_TRY(keys.alloc(std::max<uint64_t>(2 * W, 1), s));
    if (W) k_sym_keys<<<grid_for(W), kThreads, 0, s>>>(g->dag.row.p, g->dag.adj.p, rowid.p, W, lg, keys.p);
    GARY_CUDA(cudaGetLastError());
    GARY_TRY(compact_keys(keys, 2 * W, m2, s));
  }
  {
    DevBuf<uint64_t> alt;
    GARY_TRY(alt.alloc(std::max<uint64_t>(m2, 1), s));
    if (m2) GARY_TRY(radix_sort_keys(keys, alt, m2, 2 * lg, s));
  }
  GARY_TRY(padded_from_keys(keys, m2, n, lg, g->sym, s));
  GARY_CUDA(cudaStreamSynchronize(s));
  return GARY_OK;
}

int download(gary_graph *g, uint64_t *ptr, uint32_t *idx, uint32_t *perm, cudaStream_t s) {
  PaddedCSR &c = g->user_view();
  GARY_TRY(build_coo(c, s));
  std::vector<uint32_t> deg(g->n);
  GARY_CUDA(cudaMemcpyAsync(deg.data(), c.outdeg.p, (uint64_t)g->n * 4, cudaMemcpyDeviceToHost, s));
  if (idx && c.m) GARY_CUDA(cudaMemcpyAsync(idx, c.coo_col.p, c.m * 4, cudaMemcpyDeviceToHost, s));
  if (perm) {
    if (!g->keep_ids) {
      GARY_CUDA(cudaMemcpyAsync(perm, g->perm.p, (uint64_t)g->n * 4, cudaMemcpyDeviceToHost, s));
    } else {
      for (uint32_t i = 0; i < g->n; ++i) perm[i] = i;
    }
  }
  GARY_CUDA(cudaStreamSynchronize(s));
  if (ptr) {
    ptr[0] = 0;
    for (uint32_t v = 0; v < g->n; ++v) ptr[v + 1] = ptr[v] + deg[v];
  }
  return GARY_OK;
}

int csr_download(const gary_csr *c, uint64_t *ptr, uint32_t *idx) {
  if (ptr) GARY_CUDA(cudaMemcpy(ptr, c->ptr.p, ((uint64_t)c->n + 1) * 8, cudaMemcpyDeviceToHost));
  if (idx && c->nnz) GARY_CUDA(cudaMemcpy(idx, c->idx.p, c->nnz * 4, cudaMemcpyDeviceToHost));
  return GARY_OK;
}

}  // namespace gary

// C-ABI entry points for the CSR builder live here with the struct definition.
extern "C" int gary_csr_from_edges(const uint32_t *src, const uint32_t *dst, uint64_t m,
                                   uint32_t n, uint32_t flags, void *stream, gary_csr **out) {
  gary::clear_error();
  try {
    return gary::csr_from_edges(src, dst, m, n, flags, gary::as_stream(stream), out);
  } catch (const std::bad_alloc &) {
    gary::set_error("out of memory building the CSR");
    return GARY_ERR_OOM;
  } catch (const std::exception &e) {
    gary::set_error("csr_from_edges: %s", e.what());
    return GARY_ERR_CUDA;
  }
}

extern "C" int gary_csr_info(const gary_csr *c, uint32_t *n, uint64_t *nnz) {
  GARY_CHECK_ARG(c != nullptr, "csr is NULL");
  if (n) *n = c->n;
  if (nnz) *nnz = c->nnz;
  return GARY_OK;
}

extern "C" int gary_csr_device_ptrs(const gary_csr *c, const uint64_t **ptr, const uint32_t **idx) {
  GARY_CHECK_ARG(c != nullptr, "csr is NULL");
  if (ptr) *ptr = c->ptr.p;
  if (idx) *idx = c->idx.p;
  return GARY_OK;
}

extern "C" int gary_csr_download(const gary_csr *c, uint64_t *ptr, uint32_t *idx) {
  GARY_CHECK_ARG(c != nullptr, "csr is NULL");
  gary::clear_error();
  return gary::csr_download(c, ptr, idx);
}

extern "C" int gary_csr_free(gary_csr *c) {
  if (!c) return GARY_OK;
  delete c;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    gary::set_error("gary_csr_free: %s", cudaGetErrorString(e));
    return GARY_ERR_CUDA;
  }
  return GARY_OK;
}
