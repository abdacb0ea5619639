// 4-clique and 4-cycle counting.  The reference declares a second pattern
// kernel (rectCountHom, include/kernels/GraphQueryHom.cuh:48) but never
// defines it; these kernels are new, pinned by the CPU oracle and closed-form
// known answers.
//
// 4-cliques (degree-ranked DAG, every list in orientation order): each clique
// u < v < w < x is counted once at its lowest vertex u, as a triangle of the
// subgraph induced by N+(u).  For every u (d = d+(u) ids) the kernel builds
// that subgraph's upper-triangular adjacency as d bit rows of ceil(d/32)
// words: row i has bit j set when N+(u)[j] is in N+(N+(u)[i]).  Rows are
// filled by streaming each N+(v), v in N+(u), up to the largest id of N+(u)
// and looking every id up in a shared id -> position hash of N+(u).  Then
//   K4(u) = sum over set bits (i, j) of popcount(row_i AND row_j),
// since row j holds only positions after j.  Vertices with d <= 128 run on
// one warp (rows of at most 4 words), d <= 512 on a 256-thread CTA, larger
// ones on a 1024-thread CTA, with rows in shared memory up to d = 1024 and in
// a per-CTA HBM buffer beyond.
//
// 4-cycles (symmetric ranked lists): each cycle is counted once at its
// highest-ranked vertex u, with w the opposite vertex:
//   C4 = sum over u, over w < u of C(c(u,w), 2),
//   c(u,w) = |{v < u : v adjacent to u and to w}|.
// The wedges u-v-w (v, w < u) are walked and c(u,w) is accumulated in a
// counter map; adding the counter's old value at every increment sums
// C(c, 2) directly.  Three classes of u by wedge count:
//   light  (<= 512)    a warp's shared hash map;
//   medium (<= 8192)   a CTA's shared hash map;
//   heavy              dense counters in shared memory over windows of
//                      32 K consecutive w ids (16-bit counters, two to a
//                      word, three CTAs per SM).  Each v keeps a cursor into
//                      N(v) (sorted), so a window pass reads exactly the ids
//                      that fall in it; windows nothing reaches are skipped,
//                      and a heavy u is cut into tiles of consecutive windows
//                      that different CTAs take.
// All counter traffic stays in shared memory; the lists stream from HBM.
#include <thrust/binary_search.h>
#include <thrust/copy.h>
#include <thrust/count.h>
#include <thrust/execution_policy.h>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/transform_iterator.h>
#include <thrust/reduce.h>
#include <thrust/scan.h>
#include <thrust/sort.h>
#include <thrust/transform.h>
#include <thrust/transform_reduce.h>

#include <algorithm>
#include <memory>

#include "graph.cuh"
#include "patterns.cuh"
#include "warp_ops.cuh"

namespace gary {
namespace {

constexpr int kThreads = 256;
constexpr int kPWarps = 8;
constexpr uint32_t kPSlots = kC4WarpSlots;  // per-warp hash slots
static_assert(kPSlots == 1u << 10, "warp map lookups hash to 10 bits");

inline unsigned grid_for(uint64_t items) {
  uint64_t b = (items + kThreads - 1) / kThreads;
  uint64_t cap = (uint64_t)sm_count() * 16;
  return (unsigned)std::max<uint64_t>(std::min(b, cap), 1);
}

__host__ __device__ __forceinline__ uint64_t min64(uint64_t a, uint64_t b) { return a < b ? a : b; }

// ---- C4 -------------------------------------------------------------------
// Lower-ranked prefix of v's symmetric list below `u`: lower_bound(N(v), u).
__device__ __forceinline__ uint32_t prefix_below(const uint32_t *l, uint32_t len, uint32_t u) {
  uint32_t b = 0, e = len;
  while (b < e) {
    const uint32_t mid = (b + e) >> 1;
    if (l[mid] < u) b = mid + 1;
    else e = mid;
  }
  return b;
}

// |N(v) below u| for a lower neighbour v < u: N(v) (ranked, sorted) starts
// with its deg(v) - d+(v) ids below v, all below u too, so only the d+(v)
// higher ids need a search (a few probes, not log2 deg(v)).
__device__ __forceinline__ uint32_t below_u(const uint32_t *l, uint32_t len, uint32_t dplus_v, uint32_t u) {
  const uint32_t lower = len - dplus_v;
  return lower + prefix_below(l + lower, dplus_v, u);
}

// Walk every wedge u - v - w with v in N(u), v < u, and w in N(v), w < u,
// for v = N(u)[k], k in the 32-wide steps kb, kb + kstep, ... < ke; call
// f(w) for each.  All 32 lanes must call.
template <typename F>
__device__ __forceinline__ void c4_wedges(const GraphView &s, const uint32_t *__restrict__ dplus,
                                          const uint32_t *__restrict__ au, uint32_t u, uint32_t kb,
                                          uint32_t ke, uint32_t kstep, int lane, F f) {
  for (uint32_t k0 = kb; k0 < ke; k0 += kstep) {
    const uint32_t k = k0 + lane;
    uint32_t len = 0, base = 0;
    if (k < ke) {
      const uint32_t v = au[k];
      const uint2 rv = s.row[v];
      base = rv.x;
      len = (below_u(s.adj + (uint64_t)rv.x * 4, rv.y, dplus[v], u) + 3) >> 2;  // quads
    }
    const uint32_t incl = warp_inclusive_sum(len, lane);
    const uint32_t excl = incl - len;
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    const uint32_t qbase = base - excl;  // quad of flattened position p: qbase + p (mod 2^32) of the owner
    if (total == 0) continue;
    WarpRuns own(excl, len, lane);
    // one batch of quads in flight: the next loads while this one is counted
    const uint4 *adj4 = reinterpret_cast<const uint4 *>(s.adj);
    auto fetch = [&](uint32_t pb) {
      const uint32_t p = pb + lane;
      const int o = (int)own.owner(pb);
      const uint32_t qi = __shfl_sync(kFull, qbase, o) + p;
      return p < total ? adj4[qi] : make_uint4(kSentinel, kSentinel, kSentinel, kSentinel);
    };
    auto take = [&](const uint4 &a) {
      if (a.x < u) f(a.x);
      if (a.y < u) f(a.y);
      if (a.z < u) f(a.z);
      if (a.w < u) f(a.w);
    };
    uint4 cur = fetch(0);
    for (uint32_t pb = 32; pb < total; pb += 32) {
      const uint4 nxt = fetch(pb);
      take(cur);
      cur = nxt;
    }
    take(cur);
  }
}

// Counter map in shared memory: increments c(w) and returns the old value.
// The plan keeps the map at most half full; a probe that finds every slot
// taken (a broken capacity rule) sets kLaunchErrTableFull and counts nothing.
__device__ __forceinline__ uint32_t map_incr(uint32_t *keys, uint32_t *vals, uint32_t mask, int shift,
                                             uint32_t w, unsigned *err) {
  uint32_t h = (w * kHashMul) >> shift;
  for (uint32_t i = 0; i <= mask; ++i) {
    const uint32_t k = keys[h];
    if (k == w) return atomicAdd(&vals[h], 1u);
    if (k == kSentinel) {
      const uint32_t old = atomicCAS(&keys[h], kSentinel, w);
      if (old == kSentinel || old == w) return atomicAdd(&vals[h], 1u);
    }
    h = (h + 1) & mask;
  }
  atomicOr(err, kLaunchErrTableFull);
  return 0;
}

__global__ void __launch_bounds__(kPWarps * 32)
    k_c4_small(GraphView s, const uint32_t *__restrict__ dplus, const uint32_t *__restrict__ light,
               uint32_t n_light, SchedState *sched, unsigned long long *__restrict__ out) {
  extern __shared__ __align__(16) uint32_t sm[];  // kPWarps * 2 * kPSlots words
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t *keys = sm + warp * 2 * kPSlots, *vals = keys + kPSlots;
  unsigned long long acc = 0;
  while (true) {
    uint32_t c = 0;
    if (lane == 0) c = atomicAdd(&sched->next_warp, 1u);
    c = __shfl_sync(kFull, c, 0);
    const uint32_t i0 = c * 32;
    if (i0 >= n_light) break;
    const uint32_t nb = min(32u, n_light - i0);
    const uint32_t myu = lane < nb ? light[i0 + lane] : 0u;
    for (uint32_t q = 0; q < nb; ++q) {
      const uint32_t u = __shfl_sync(kFull, myu, q);
      const uint2 ru = s.row[u];
      const uint32_t pre = ru.y - dplus[u];  // neighbours ranked below u
      const uint32_t *au = s.adj + (uint64_t)ru.x * 4;
      for (uint32_t i = lane; i < kPSlots; i += 32) {
        keys[i] = kSentinel;
        vals[i] = 0;
      }
      __syncwarp();
      c4_wedges(s, dplus, au, u, 0, pre, 32, lane, [&](uint32_t w) {
        acc += map_incr(keys, vals, kPSlots - 1, 32 - 10, w, &sched->error);
      });
      __syncwarp();
    }
  }
  acc = warp_sum_u64(acc);
  if (lane == 0 && acc) atomicAdd(out, acc);
}

// ---- C4, medium vertices: one CTA-wide shared hash map per vertex ---------
// A count c(u,w) never exceeds the vertex's wedge count (each v adds at most
// one to it), at most kMidWedges here, so counts are 16 bits, two to a word:
// keys 64 KiB + counts 32 KiB, and two CTAs share an SM.
constexpr uint32_t kMidSlots = kC4MidSlots;
constexpr int kMidLog = 14;
static_assert((1u << kMidLog) == kMidSlots, "medium map size");
constexpr int kMidThreads = 512;
constexpr uint64_t kMidWedges = kC4MidWedges;  // wedges (>= distinct w) a medium vertex may have
constexpr uint32_t kMidWords = kMidSlots + kMidSlots / 2;
static_assert(kMidWedges < 65536, "16-bit medium counts");

// As map_incr, with the count of slot h in half h & 1 of word h / 2 of vals2.
__device__ __forceinline__ uint32_t map_incr16(uint32_t *keys, uint32_t *vals2, uint32_t mask, int shift,
                                               uint32_t w, unsigned *err) {
  uint32_t h = (w * kHashMul) >> shift;
  for (uint32_t i = 0; i <= mask; ++i) {
    const uint32_t k = keys[h];
    bool hit = k == w;
    if (!hit && k == kSentinel) {
      const uint32_t old = atomicCAS(&keys[h], kSentinel, w);
      hit = old == kSentinel || old == w;
    }
    if (hit) {
      const uint32_t sh = (h & 1u) << 4;
      return (atomicAdd(&vals2[h >> 1], 1u << sh) >> sh) & 0xFFFFu;
    }
    h = (h + 1) & mask;
  }
  atomicOr(err, kLaunchErrTableFull);
  return 0;
}

__global__ void __launch_bounds__(kMidThreads, 2)
    k_c4_mid(GraphView s, const uint32_t *__restrict__ dplus, const uint32_t *__restrict__ mid,
             uint32_t n_mid, SchedState *sched, unsigned long long *__restrict__ out) {
  extern __shared__ __align__(16) uint32_t sm[];
  uint32_t *keys = sm, *vals = sm + kMidSlots;  // vals: kMidSlots / 2 words of 16-bit pairs
  __shared__ uint32_t s_u, s_next;
  const int lane = threadIdx.x & 31;
  unsigned long long acc = 0;
  for (uint32_t i = threadIdx.x; i < kMidSlots; i += blockDim.x) keys[i] = kSentinel;
  for (uint32_t i = threadIdx.x; i < kMidSlots / 2; i += blockDim.x) vals[i] = 0;
  while (true) {
    if (threadIdx.x == 0) {
      s_u = atomicAdd(&sched->next_aux, 1u);
      s_next = 0;
    }
    __syncthreads();
    if (s_u >= n_mid) break;
    const uint32_t u = mid[s_u];
    const uint2 ru = s.row[u];
    const uint32_t pre = ru.y - dplus[u];
    const uint32_t *au = s.adj + (uint64_t)ru.x * 4;
    while (true) {
      uint32_t k = 0;
      if (lane == 0) k = atomicAdd(&s_next, 32u);
      k = __shfl_sync(kFull, k, 0);
      if (k >= pre) break;
      c4_wedges(s, dplus, au, u, k, min(k + 32, pre), 32, lane, [&](uint32_t w) {
        acc += map_incr16(keys, vals, kMidSlots - 1, 32 - kMidLog, w, &sched->error);
      });
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < kMidSlots; i += blockDim.x) keys[i] = kSentinel;
    for (uint32_t i = threadIdx.x; i < kMidSlots / 2; i += blockDim.x) vals[i] = 0;
    // the loop head's barrier orders this reset before the next vertex
  }
  acc = warp_sum_u64(acc);
  if (lane == 0 && acc) atomicAdd(out, acc);
}

// ---- C4, heavy vertices: dense counters over windows of w ids ---------------
// A window is kWinIds consecutive w ids; its counters take kWinWords shared
// words (64 KiB), so three 512-thread CTAs share an SM and the others run
// while one waits at a barrier (measured at RMAT-22 / RMAT-24: 48 K ids with
// two CTAs per SM 260 ms / 5.53 s, 32 K ids with three 225 ms / 4.88 s,
// 24 K ids with four 256-thread CTAs 317 ms / 7.57 s).  A counter never
// exceeds pre(u), the number of lower neighbours of u, so for pre(u) < 2^16
// two 16-bit counters share a word and a whole window fits; otherwise the
// window is counted in two halves of kWinWords 32-bit counters.
constexpr uint32_t kWinIds = 32 * 1024;
constexpr uint32_t kWinWords = 16 * 1024;
constexpr int kWinThreads = 512;
constexpr int kWinWarps = kWinThreads / 32;

__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t *l, uint32_t b, uint32_t e,
                                                    uint32_t x) {
  while (b < e) {
    const uint32_t m = (b + e) >> 1;
    if (l[m] < x) b = m + 1;
    else e = m;
  }
  return b;
}

// First index i in [c, len) with l[i] >= x (len when none), galloping from c:
// cheap when the answer is near c, as it is for a cursor moving one window on.
__device__ __forceinline__ uint32_t gallop_geq(const uint32_t *l, uint32_t c, uint32_t len,
                                               uint32_t x) {
  if (c >= len || l[c] >= x) return c;
  uint32_t b = c, step = 1;  // l[b] < x
  while ((uint64_t)b + step < len && l[b + step] < x) {
    b += step;
    step <<= 1;
  }
  const uint64_t e = (uint64_t)b + step < len ? (uint64_t)b + step : len;
  return lower_bound_u32(l, b + 1, (uint32_t)e, x);
}

// The same answer for a list in the padded layout (32-byte aligned, padded
// with kSentinel to a multiple of 8): the 16 ids of the two octets from c's
// octet come in one round of loads and settle most runs (70 % of a window's
// runs hold at most 8 ids); only a run that goes past them gallops on.
__device__ __forceinline__ uint32_t run_end(const uint32_t *l, uint32_t c, uint32_t len, uint32_t x,
                                            uint32_t *at_end = nullptr) {
  if (c >= len) {
    if (at_end) *at_end = kSentinel;
    return c;
  }
  const uint32_t ob = c & ~7u;
  const uint32_t plen = (len + 7u) & ~7u;
  const uint4 *q = reinterpret_cast<const uint4 *>(l + ob);
  const uint4 s4 = make_uint4(kSentinel, kSentinel, kSentinel, kSentinel);
  const uint4 a0 = q[0], a1 = q[1];
  const bool two = ob + 8 < plen;
  const uint4 b0 = two ? q[2] : s4, b1 = two ? q[3] : s4;
  const uint32_t id[16] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w,
                           b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
  uint32_t e = kSentinel, ide = kSentinel;
#pragma unroll
  for (int i = 15; i >= 0; --i)
    if (ob + i >= c && (ob + i >= len || id[i] >= x)) {
      e = ob + i;
      ide = ob + i < len ? id[i] : kSentinel;
    }
  if (e == kSentinel) {
    e = gallop_geq(l, ob + 16, len, x);  // ids [c, ob + 16) are all below x
    ide = e < len ? l[e] : kSentinel;
  }
  if (at_end) *at_end = ide;  // the id at e (kSentinel at the end of the list)
  return e;
}

__device__ __forceinline__ uint32_t warp_min_u32(uint32_t x) {
#pragma unroll
  for (int o = 16; o; o >>= 1) x = min(x, __shfl_xor_sync(kFull, x, o));
  return x;
}

// Walk, for the 32 list ranges [b_k, e_k) of the lanes' v's, every id w of
// N(v_k) in that range; call f(w).  The ranges are read as the 16-byte quads
// of the (16-byte aligned, sorted, padded) lists that cover them, flattened
// across the lanes; a quad's other ids lie below lo (before the range) or at
// or past lo + span (after it, or padding), so the window's own range test
// rejects them.  All lanes call.  The ranges of the active neighbours are
// never empty (each has an id in the window) and the lanes past the active
// list come last, so the owners follow from the starts (WarpOwners).
template <typename F>
__device__ __forceinline__ void walk_ranges(const uint32_t *__restrict__ adj, uint32_t q4, uint32_t b,
                                            uint32_t e, uint32_t lo, uint32_t span, int lane, F f) {
  const uint32_t nq = e > b ? ((e + 3) >> 2) - (b >> 2) : 0u;
  const uint32_t incl = warp_inclusive_sum(nq, lane);
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  if (total == 0) return;
  // quad of flattened position p: qbase + p (mod 2^32) of the owner
  const uint32_t qbase = q4 + (b >> 2) - (incl - nq);
  WarpOwners own(incl - nq, lane);
  const uint4 *adj4 = reinterpret_cast<const uint4 *>(adj);
  auto fetch = [&](uint32_t pb) {
    const uint32_t p = pb + lane;
    const int o = (int)own.owner(pb);
    const uint32_t qi = __shfl_sync(kFull, qbase, o) + p;
    return p < total ? adj4[qi] : make_uint4(kSentinel, kSentinel, kSentinel, kSentinel);
  };
  auto take = [&](const uint4 &a) {
    if (a.x - lo < span) f(a.x);
    if (a.y - lo < span) f(a.y);
    if (a.z - lo < span) f(a.z);
    if (a.w - lo < span) f(a.w);
  };
  uint4 cur = fetch(0);
  for (uint32_t pb = 32; pb < total; pb += 32) {
    const uint4 nxt = fetch(pb);
    take(cur);
    cur = nxt;
  }
  take(cur);
}

// Tile {v0 = u, v1 = pre, j0 = wa, j1 = wb}: windows [wa, wb) of vertex u,
// i.e. wedge ends w in [wa * kWinIds, min(wb * kWinIds, u)).  The kernel
// steps through them in passes of ws ids: kWinIds with 16-bit counters,
// kWinIds / 2 with 32-bit ones.
//
// Per lower neighbour k (v = N(u)[k]) the CTA keeps, in its HBM scratch, v's
// row record, a cursor into N(v), the cursor before the last pass, and the
// pass index of the id at the cursor (nextw).  A pass scans nextw, compacts
// the neighbours whose next id falls in it into an active list, and only
// those walk; the scan also yields the next non-empty pass.  Neighbours with
// few ids below u are active in few passes, so most passes touch a small part
// of the list.
constexpr uint32_t kNoWindow = 0xFFFFFFFFu;

struct C4Scratch {
  uint2 *vrow;     // row record of each lower neighbour
  uint32_t *cur, *prev, *nextw, *act;
};

__device__ __forceinline__ C4Scratch c4_scratch(uint32_t *base, uint32_t max_pre) {
  C4Scratch c;
  c.vrow = reinterpret_cast<uint2 *>(base);
  c.cur = base + 2 * (uint64_t)max_pre;
  c.prev = c.cur + max_pre;
  c.nextw = c.prev + max_pre;
  c.act = c.nextw + max_pre;
  return c;
}

// words of scratch per lower neighbour (vrow 2, cur, prev, nextw, act)
constexpr uint32_t kC4ScratchWords = 6;

// Counter of w (offset o = w - lo in the pass) incremented; returns its old value.
template <bool WIDE>
__device__ __forceinline__ uint32_t win_incr(uint32_t *cnt, uint32_t o) {
  if (WIDE) return atomicAdd(&cnt[o], 1u);
  const uint32_t sh = (o & 1u) << 4;
  return (atomicAdd(&cnt[o >> 1], 1u << sh) >> sh) & 0xFFFFu;
}

__global__ void __launch_bounds__(kWinThreads, 3)
    k_c4_win(GraphView s, const Tile *__restrict__ tiles, uint32_t t_lo, uint32_t t_hi,
             uint32_t *__restrict__ scratch, uint32_t max_pre, SchedState *sched,
             unsigned long long *__restrict__ out) {
  extern __shared__ __align__(16) uint32_t cnt[];  // kWinWords words, zero between passes
  __shared__ uint32_t s_tile, s_next, s_nact, s_minw;
  __shared__ unsigned long long s_wedges;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const C4Scratch cs = c4_scratch(scratch + (uint64_t)blockIdx.x * kC4ScratchWords * max_pre, max_pre);
  unsigned long long acc = 0;
  for (uint32_t i = threadIdx.x; i < kWinWords; i += blockDim.x) cnt[i] = 0;
  while (true) {
    if (threadIdx.x == 0) {
      s_tile = t_lo + atomicAdd(&sched->next_cta, 1u);
      s_minw = kNoWindow;
    }
    __syncthreads();
    const uint32_t t = s_tile;
    if (t >= t_hi) break;
    const Tile tl = tiles[t];
    const uint32_t u = tl.v0, pre = tl.v1;
    const bool wide = c4_wide_counters(pre);
    const uint32_t ws = wide ? kWinIds / 2 : kWinIds;  // ids per pass
    const uint32_t *au = s.adj + (uint64_t)s.row[u].x * 4;
    const uint64_t end64 = (uint64_t)tl.j1 * kWinIds, begin64 = (uint64_t)tl.j0 * kWinIds;
    const uint32_t w_end = end64 < u ? (uint32_t)end64 : u;
    const uint32_t w_begin = begin64 < w_end ? (uint32_t)begin64 : w_end;
    // state at the tile's first pass
    uint32_t mw = kNoWindow;
    for (uint32_t k = threadIdx.x; k < pre; k += blockDim.x) {
      const uint2 rv = s.row[au[k]];
      const uint32_t *l = s.adj + (uint64_t)rv.x * 4;
      const uint32_t c = w_begin ? lower_bound_u32(l, 0, rv.y, w_begin) : 0u;
      const uint32_t x = c < rv.y ? l[c] : kSentinel;
      const uint32_t nw = x < w_end ? x / ws : kNoWindow;
      cs.vrow[k] = rv;
      cs.cur[k] = c;
      cs.nextw[k] = nw;
      mw = min(mw, nw);
    }
    mw = warp_min_u32(mw);
    if (lane == 0) atomicMin(&s_minw, mw);
    __syncthreads();
    while (true) {
      const uint32_t win = s_minw;
      if (win == kNoWindow) break;  // no id of the tile's range is left
      const uint32_t lo = win * ws;
      const uint32_t hi = lo + ws < w_end ? lo + ws : w_end;
      __syncthreads();  // every thread has read s_minw
      if (threadIdx.x == 0) {
        s_next = 0;
        s_nact = 0;
        s_minw = kNoWindow;
        s_wedges = 0;
      }
      __syncthreads();
      // active neighbours of this pass; the others keep their next pass
      uint32_t mwi = kNoWindow;
      for (uint32_t k0 = warp * 32; k0 < pre; k0 += kWinThreads) {
        const uint32_t k = k0 + lane;
        const uint32_t nw = k < pre ? cs.nextw[k] : kNoWindow;
        const bool on = nw == win;
        const unsigned m = __ballot_sync(kFull, on);
        uint32_t at = 0;
        if (lane == 0 && m) at = atomicAdd(&s_nact, (uint32_t)__popc(m));
        at = __shfl_sync(kFull, at, 0);
        if (on) cs.act[at + __popc(m & ((1u << lane) - 1u))] = k;
        else mwi = min(mwi, nw);
      }
      mwi = warp_min_u32(mwi);
      if (lane == 0) atomicMin(&s_minw, mwi);
      __syncthreads();
      const uint32_t nact = s_nact;
      // count: advance the active cursors past the pass, counting the ids passed
      uint32_t nxt = kNoWindow;
      unsigned long long seen = 0;
      while (true) {
        uint32_t k0 = 0;
        if (lane == 0) k0 = atomicAdd(&s_next, 32u);
        k0 = __shfl_sync(kFull, k0, 0);
        if (k0 >= nact) break;
        const uint32_t a = k0 + lane;
        uint32_t q4 = 0, b = 0, e = 0;
        if (a < nact) {
          const uint32_t k = cs.act[a];
          const uint2 rv = cs.vrow[k];
          const uint32_t *l = s.adj + (uint64_t)rv.x * 4;
          b = cs.cur[k];
          uint32_t x;
          e = run_end(l, b, rv.y, hi, &x);
          cs.prev[k] = b;
          cs.cur[k] = e;
          const uint32_t nw = x < w_end ? x / ws : kNoWindow;
          cs.nextw[k] = nw;
          nxt = min(nxt, nw);
          q4 = rv.x;
          seen += e - b;
        }
        if (wide)
          walk_ranges(s.adj, q4, b, e, lo, hi - lo, lane, [&](uint32_t w) { acc += win_incr<true>(cnt, w - lo); });
        else
          walk_ranges(s.adj, q4, b, e, lo, hi - lo, lane, [&](uint32_t w) { acc += win_incr<false>(cnt, w - lo); });
      }
      nxt = warp_min_u32(nxt);
      seen = warp_sum_u64(seen);
      if (lane == 0) {
        atomicMin(&s_minw, nxt);
        if (seen) atomicAdd(&s_wedges, seen);
      }
      __syncthreads();
      // zero the pass's counters again: walk the same ids when few, else clear them whole
      const uint32_t words = wide ? hi - lo : (hi - lo + 1) >> 1;
      if (s_wedges + nact < words / 4) {
        for (uint32_t a0 = warp * 32; a0 < nact; a0 += kWinWarps * 32) {
          const uint32_t a = a0 + lane;
          uint32_t q4 = 0, b = 0, e = 0;
          if (a < nact) {
            const uint32_t k = cs.act[a];
            q4 = cs.vrow[k].x;
            b = cs.prev[k];
            e = cs.cur[k];
          }
          walk_ranges(s.adj, q4, b, e, lo, hi - lo, lane, [&](uint32_t w) { cnt[wide ? w - lo : (w - lo) >> 1] = 0u; });
        }
      } else {
        for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) cnt[i] = 0;
      }
      __syncthreads();
    }
  }
  acc = warp_sum_u64(acc);
  if (lane == 0 && acc) atomicAdd(out, acc);
}

// ---- K4: bit rows of the subgraph induced by N+(u) -------------------------
// Three sizes of worker, so that no worker waits at barriers it does not need:
//   warp vertices (3 <= d+ <= 128): one warp each, 8-warp CTAs, several per SM;
//   mid vertices (128 < d+ <= 362): a 256-thread CTA each, rows in 17 KiB of
//     shared memory, eight CTAs per SM (one waits at a barrier, others run);
//   big vertices (d+ > 362): a 1024-thread CTA each, two per SM: rows in 96
//     KiB of shared memory up to d+ = 877; beyond, rows in a per-CTA HBM buffer
//     and only the position hash in shared memory (k_k4_pool, run first: its
//     vertices are the largest).
// (class bounds, table sizes and row words: pattern_rules.cuh)
constexpr uint32_t kK4WarpWords = 1024;       // shared words per warp: 32 KiB per CTA, up to 7 CTAs per SM
constexpr int kK4WarpCtaWarps = 8;
constexpr int kK4MidThreads = 256;
constexpr int kK4BigThreads = 1024;
constexpr uint32_t kK4PoolPerSm = 2;         // CTAs per SM of the HBM-row kernel
static_assert(2 * (1u << kK4WarpLog) + kK4WarpRowWords <= kK4WarpWords, "warp region too small");

// Position hash of N+(u) (ids are distinct).  k4_vertex inserts at most
// half as many ids as the table has slots, so every lookup ends at a free
// slot and needs no counter (a counter cost the hot lookup about 13 %).  The
// insert loop visits each slot at most once regardless.
__device__ __forceinline__ void pos_insert(uint32_t *keys, uint32_t *pos, uint32_t mask, int shift,
                                           uint32_t x, uint32_t p, unsigned *err) {
  uint32_t h = (x * kHashMul) >> shift;
  for (uint32_t i = 0; i <= mask; ++i) {
    if (atomicCAS(&keys[h], kSentinel, x) == kSentinel) {
      pos[h] = p;
      return;
    }
    h = (h + 1) & mask;
  }
  atomicOr(err, kLaunchErrTableFull);
}

__device__ __forceinline__ int pos_find(const uint32_t *keys, const uint32_t *pos, uint32_t mask,
                                        int shift, uint32_t x) {
  uint32_t h = (x * kHashMul) >> shift;
  while (true) {
    const uint32_t k = keys[h];
    if (k == kSentinel) return -1;  // first: x may itself be the padding value
    if (k == x) return (int)pos[h];
    h = (h + 1) & mask;
  }
}

// 4-cliques with lowest vertex u; `nthreads` threads (one warp or the CTA)
// cooperate, separated by sync().  On entry and on return every key slot of
// the hash holds kSentinel and the d * W row words are zero.
template <typename Sync>
__device__ unsigned long long k4_vertex(const GraphView &g, uint32_t u, uint32_t *keys, uint32_t *pos,
                                        uint32_t max_log, uint32_t *rows, uint32_t tid,
                                        uint32_t nthreads, Sync sync, unsigned *err) {
  const int lane = tid & 31;
  const uint2 ru = g.row[u];
  const uint32_t d = ru.y;
  const uint32_t *au = g.adj + (uint64_t)ru.x * 4;
  const uint32_t W = (d + 31) >> 5;
  int l = hash_log2(d);
  if (l > (int)max_log) l = (int)max_log;
  const uint32_t mask = (1u << l) - 1;
  const int shift = 32 - l;
  // at most half the slots: the plan's degree classes keep d there; a list
  // beyond that (a broken rule) is counted wrongly but reported, never hangs
  const uint32_t ins = d <= (mask + 1) / 2 ? d : (mask + 1) / 2;
  if (ins < d && tid == 0) atomicOr(err, kLaunchErrTableFull);
  for (uint32_t i = tid; i < ins; i += nthreads) pos_insert(keys, pos, mask, shift, au[i], i, err);
  sync();
  const uint32_t maxu = au[d - 1];
  // rows: 32 rows per warp step.  Each N+(v) is read as 32-byte octets from
  // its (32-byte aligned, padded) start up to the last id <= max N+(u); the
  // lanes walk the 32 lists' octets flattened.  Ids past that point (larger
  // ids, padding) are not in N+(u), so the hash rejects them: no mask.
  const uint4 *adj4 = reinterpret_cast<const uint4 *>(g.adj);
  auto mark = [&](uint32_t row, uint32_t x) {
    const int j = pos_find(keys, pos, mask, shift, x);
    if (j >= 0) atomicOr(&rows[row * W + ((uint32_t)j >> 5)], 1u << (j & 31));
  };
  for (uint32_t r0 = tid & ~31u; r0 < d; r0 += nthreads) {
    const uint32_t i = r0 + lane;
    uint32_t o0 = 0, no = 0;
    if (i < d) {
      const uint2 rv = g.row[au[i]];
      const uint32_t e = prefix_below(g.adj + (uint64_t)rv.x * 4, rv.y, maxu + 1);  // ids <= max N+(u)
      o0 = rv.x >> 1;
      no = (e + 7) >> 3;
    }
    const uint32_t incl = warp_inclusive_sum(no, lane);
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    const uint32_t bias = o0 - (incl - no);
    WarpRuns own(incl - no, no, lane);
    for (uint32_t pb = 0; pb < total; pb += 32) {
      const uint32_t p = pb + lane;
      const int o = (int)own.owner(pb);
      const uint32_t oc = __shfl_sync(kFull, bias, o) + p;
      if (p < total) {
        const uint4 a = adj4[2 * (uint64_t)oc], b = adj4[2 * (uint64_t)oc + 1];
        const uint32_t row = r0 + o;
        mark(row, a.x); mark(row, a.y); mark(row, a.z); mark(row, a.w);
        mark(row, b.x); mark(row, b.y); mark(row, b.z); mark(row, b.w);
      }
    }
  }
  sync();
  // count: for every set bit (i, j), the common later positions of rows i and j
  unsigned long long cnt = 0;
  for (uint32_t it = tid; it < d * W; it += nthreads) {
    const uint32_t i = it / W, w = it - i * W;
    const uint32_t *ri = rows + i * W;
    uint32_t bits = ri[w];
    while (bits) {
      const uint32_t j = w * 32 + (__ffs(bits) - 1);
      bits &= bits - 1;
      const uint32_t *rj = rows + j * W;
      for (uint32_t ww = w; ww < W; ++ww) cnt += __popc(ri[ww] & rj[ww]);
    }
  }
  sync();
  for (uint32_t it = tid; it < d * W; it += nthreads) rows[it] = 0;
  for (uint32_t h = tid; h <= mask; h += nthreads) keys[h] = kSentinel;
  sync();
  return cnt;
}

// One listed vertex per CTA at a time, claimed through *counter.  ROWW = 0:
// every vertex keeps its rows in its CTA's HBM buffer, and the CTA holds only
// the position hash in shared memory.
template <int THREADS, int HLOG, uint32_t ROWW>
__device__ __forceinline__ void k4_cta_body(GraphView g, const uint32_t *__restrict__ list, uint32_t lo,
                                            uint32_t hi, uint32_t *__restrict__ pool, uint64_t pool_words,
                                            uint32_t *counter, unsigned *err,
                                            unsigned long long *__restrict__ out) {
  extern __shared__ __align__(16) uint32_t sm[];
  __shared__ uint32_t s_idx;
  uint32_t *keys = sm, *pos = sm + (1u << HLOG), *srows = sm + 2 * (1u << HLOG);
  for (uint32_t i = threadIdx.x; i < (1u << HLOG); i += blockDim.x) keys[i] = kSentinel;
  for (uint32_t i = threadIdx.x; i < ROWW; i += blockDim.x) srows[i] = 0;
  unsigned long long cnt = 0;
  while (true) {
    if (threadIdx.x == 0) s_idx = lo + atomicAdd(counter, 1u);
    __syncthreads();
    const uint32_t k = s_idx;
    __syncthreads();  // every thread has read s_idx
    if (k >= hi) break;
    const uint32_t u = list[k];
    const uint32_t d = g.row[u].y;
    const uint64_t words = (uint64_t)d * ((d + 31) >> 5);
    uint32_t *rows = words <= ROWW ? srows : pool + (uint64_t)blockIdx.x * pool_words;
    cnt += k4_vertex(g, u, keys, pos, HLOG, rows, threadIdx.x, blockDim.x, [] { __syncthreads(); }, err);
  }
  cnt = warp_sum_u64(cnt);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(out, cnt);
}

template <int THREADS, int HLOG, uint32_t ROWW>
__global__ void __launch_bounds__(THREADS)
    k_k4_cta(GraphView g, const uint32_t *__restrict__ list, uint32_t lo, uint32_t hi,
             uint32_t *__restrict__ pool, uint64_t pool_words, uint32_t *counter, unsigned *err,
             unsigned long long *__restrict__ out) {
  k4_cta_body<THREADS, HLOG, ROWW>(g, list, lo, hi, pool, pool_words, counter, err, out);
}

// Vertices whose rows live in HBM: two 1024-thread CTAs share an SM.
__global__ void __launch_bounds__(kK4BigThreads, kK4PoolPerSm)
    k_k4_pool(GraphView g, const uint32_t *__restrict__ list, uint32_t lo, uint32_t hi,
              uint32_t *__restrict__ pool, uint64_t pool_words, uint32_t *counter, unsigned *err,
              unsigned long long *__restrict__ out) {
  k4_cta_body<kK4BigThreads, kK4PoolLog, 0>(g, list, lo, hi, pool, pool_words, counter, err, out);
}

// Warp vertices: each warp in its own region of shared memory, one vertex per
// claim (32 per claim left a tail of costly vertices: RMAT-22 129.1 -> 119.6 ms).
__global__ void __launch_bounds__(kK4WarpCtaWarps * 32)
    k_k4_warp(GraphView g, const uint32_t *__restrict__ list, uint32_t lo, uint32_t hi,
              uint32_t *counter, unsigned *err, unsigned long long *__restrict__ out) {
  extern __shared__ __align__(16) uint32_t sm[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t *keys = sm + warp * kK4WarpWords, *pos = keys + (1u << kK4WarpLog),
           *rows = pos + (1u << kK4WarpLog);
  for (uint32_t i = lane; i < (1u << kK4WarpLog); i += 32) keys[i] = kSentinel;
  for (uint32_t i = lane; i < kK4WarpMaxD * (kK4WarpMaxD / 32); i += 32) rows[i] = 0;
  __syncwarp();
  unsigned long long cnt = 0;
  while (true) {
    uint32_t c = 0;
    if (lane == 0) c = atomicAdd(counter, 1u);
    c = __shfl_sync(kFull, c, 0);
    if (lo + c >= hi) break;
    cnt += k4_vertex(g, list[lo + c], keys, pos, kK4WarpLog, rows, lane, 32, [] { __syncwarp(); }, err);
  }
  cnt = warp_sum_u64(cnt);
  if (lane == 0 && cnt) atomicAdd(out, cnt);
}

// ---- plans ------------------------------------------------------------------
struct ClassIs {
  const uint8_t *cls;
  uint8_t c;
  __host__ __device__ bool operator()(uint32_t v) const { return cls[v] == c; }
};
// C4 per-vertex class by an upper bound of its wedge count.
__global__ void k_c4_classify(const uint2 *__restrict__ srow, const uint32_t *__restrict__ sadj,
                              const uint32_t *__restrict__ dplus, uint32_t n, uint32_t warp_cap,
                              uint8_t *__restrict__ cls) {
  for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n;
       u += (uint64_t)gridDim.x * blockDim.x) {
    const uint2 r = srow[u];
    const uint32_t pre = r.y - dplus[u];
    uint64_t w = 0;
    for (uint32_t k = 0; k < pre && w <= warp_cap; ++k) w += srow[sadj[(uint64_t)r.x * 4 + k]].y;
    // w: the wedge bound, its sum stopped once past the light limit; the
    // exact counts that split the others come later
    const C4Class c = c4_class(pre, w, ~0ull);
    cls[u] = c == kC4None ? kClassNone : (c == kC4Light ? kClassLight : kClassCta);
  }
}

// Exact wedge count of each listed vertex: sum over v in N(u), v < u, of
// |N(v) below u|.  One warp per vertex.
__global__ void k_c4_exact_wedges(const uint2 *__restrict__ srow, const uint32_t *__restrict__ sadj,
                                  const uint32_t *__restrict__ dplus, const uint32_t *__restrict__ list,
                                  uint32_t nl, uint64_t *__restrict__ wed) {
  const int lane = threadIdx.x & 31;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nl; i += warps) {
    const uint32_t u = list[i];
    const uint2 ru = srow[u];
    const uint32_t pre = ru.y - dplus[u];
    uint64_t w = 0;
    for (uint32_t k = lane; k < pre; k += 32) {
      const uint32_t v = sadj[(uint64_t)ru.x * 4 + k];
      const uint2 rv = srow[v];
      w += below_u(sadj + (uint64_t)rv.x * 4, rv.y, dplus[v], u);
    }
    w = warp_sum_u64(w);
    if (lane == 0) wed[i] = w;
  }
}

__host__ __device__ __forceinline__ uint32_t c4_windows(uint32_t u) {
  return (uint32_t)(((uint64_t)u + kWinIds - 1) / kWinIds);
}

// Cost of a heavy vertex in probe units: its wedges, a cursor step per
// (window, v), a barrier-bound overhead per window.
__global__ void k_c4_heavy_cost(const uint2 *__restrict__ srow, const uint32_t *__restrict__ dplus,
                                const uint32_t *__restrict__ heavy, const uint64_t *__restrict__ wed,
                                uint32_t nh, uint64_t *__restrict__ cost) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nh;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t u = heavy[i];
    const uint32_t pre = srow[u].y - dplus[u];
    const uint64_t nw = c4_windows(u);
    cost[i] = wed[i] + nw * (2ull * pre + 4096);
  }
}

__global__ void k_c4_tile_counts(const uint32_t *__restrict__ heavy, const uint64_t *__restrict__ cost,
                                 uint32_t nh, uint64_t target, uint32_t *__restrict__ kt) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nh;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t want = (cost[i] + target - 1) / target;
    const uint64_t nw = c4_windows(heavy[i]);
    kt[i] = (uint32_t)(want < 1 ? 1 : (want > nw ? nw : want));
  }
}

__global__ void k_c4_fill_tiles(const uint2 *__restrict__ srow, const uint32_t *__restrict__ dplus,
                                const uint32_t *__restrict__ heavy, uint32_t nh,
                                const uint32_t *__restrict__ off, Tile *__restrict__ tiles) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nh;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t u = heavy[i];
    const uint32_t pre = srow[u].y - dplus[u];
    const uint32_t kk = off[i + 1] - off[i];
    const uint64_t nw = c4_windows(u);
    for (uint32_t j = 0; j < kk; ++j) {
      Tile t;
      t.v0 = u;
      t.v1 = pre;
      t.j0 = (uint32_t)(nw * j / kk);
      t.j1 = (uint32_t)(nw * (j + 1) / kk);
      tiles[off[i] + j] = t;
    }
  }
}

struct K4WorkerIn {
  const uint32_t *d;
  K4Worker lo, hi;
  __host__ __device__ bool operator()(uint32_t u) const {
    const K4Worker w = k4_worker(d[u]);
    return w >= lo && w <= hi;
  }
};
struct DegOf {
  const uint32_t *d;
  __host__ __device__ uint32_t operator()(uint32_t u) const { return d[u]; }
};
struct AtMost {
  uint64_t cap;
  __host__ __device__ bool operator()(uint64_t w) const { return w <= cap; }
};
struct Above {
  uint64_t cap;
  __host__ __device__ bool operator()(uint64_t w) const { return w > cap; }
};
struct PreOf {
  const uint2 *srow;
  const uint32_t *dplus;
  __host__ __device__ uint32_t operator()(uint32_t u) const { return srow[u].y - dplus[u]; }
};
struct K4PoolDegree {
  __host__ __device__ bool operator()(uint32_t d) const { return k4_worker(d) == kK4Pool; }
};
struct MaxU32 {
  __host__ __device__ uint32_t operator()(uint32_t a, uint32_t b) const { return a > b ? a : b; }
};

}  // namespace

// ---------------------------------------------------------------------------
// The window kernel's shared-memory opt-in, once per device.
int c4_win_attr() {
  static bool done[64] = {false};
  const int dev = device_ordinal();
  if (dev < 64 && done[dev]) return GARY_OK;
  GARY_CUDA(cudaFuncSetAttribute(k_c4_win, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(kWinWords * 4)));
  if (dev < 64) done[dev] = true;
  return GARY_OK;
}

int build_k4_plan(gary_graph *g, cudaStream_t s, PatternPlan **out) {
  auto plan = std::make_unique<PatternPlan>();
  const uint32_t n = g->n;
  ScratchAlloc pol_alloc{s};
  auto pol = thrust::cuda::par_nosync(pol_alloc).on(s);
  const uint32_t *dp = g->dag.outdeg.p;
  // warp and mid vertices in id order; big vertices largest first
  GARY_TRY(plan->light.alloc_persistent(std::max<uint32_t>(n, 1)));
  plan->n_light = (uint32_t)(thrust::copy_if(pol, thrust::counting_iterator<uint32_t>(0),
                                             thrust::counting_iterator<uint32_t>(n), plan->light.p,
                                             K4WorkerIn{dp, kK4Warp, kK4Warp}) - plan->light.p);
  GARY_TRY(plan->mid.alloc_persistent(std::max<uint32_t>(n, 1)));
  plan->n_mid = (uint32_t)(thrust::copy_if(pol, thrust::counting_iterator<uint32_t>(0),
                                           thrust::counting_iterator<uint32_t>(n), plan->mid.p,
                                           K4WorkerIn{dp, kK4Mid, kK4Mid}) - plan->mid.p);
  GARY_TRY(plan->big.alloc_persistent(std::max<uint32_t>(n, 1)));
  plan->n_big = (uint32_t)(thrust::copy_if(pol, thrust::counting_iterator<uint32_t>(0),
                                           thrust::counting_iterator<uint32_t>(n), plan->big.p,
                                           K4WorkerIn{dp, kK4Big, kK4Pool}) - plan->big.p);
  if (plan->n_big) {
    DevBuf<uint32_t> key;
    GARY_TRY(key.alloc(plan->n_big, s));
    thrust::transform(pol, plan->big.p, plan->big.p + plan->n_big, key.p, DegOf{dp});
    thrust::sort_by_key(pol, key.p, key.p + plan->n_big, plan->big.p, thrust::greater<uint32_t>());
    uint32_t dmax = 0;
    GARY_CUDA(cudaMemcpyAsync(&dmax, key.p, 4, cudaMemcpyDeviceToHost, s));
    GARY_CUDA(cudaStreamSynchronize(s));
    plan->max_pre = dmax;
    plan->n_pool = (uint32_t)thrust::count_if(pol, key.p, key.p + plan->n_big, K4PoolDegree{});
    plan->win_ctas = (uint32_t)sm_count() * kK4PoolPerSm;
    const uint64_t words = (uint64_t)dmax * ((dmax + 31) / 32);
    if (plan->n_pool) {  // rows of the largest vertices live in HBM, one buffer per CTA
      GARY_TRY(plan->cursors.alloc_persistent((uint64_t)plan->win_ctas * words));
      GARY_CUDA(cudaMemsetAsync(plan->cursors.p, 0, plan->cursors.bytes(), s));
    }
  }
  GARY_TRY(plan->sched.alloc_persistent(1));
  GARY_CUDA(cudaStreamSynchronize(s));
  *out = plan.release();
  return GARY_OK;
}

int launch_k4(gary_graph *g, PatternPlan *plan, unsigned long long *d_out, cudaStream_t s,
              uint32_t shard, uint32_t nshards) {
  auto part = [&](uint32_t total, uint32_t k) { return (uint32_t)((uint64_t)total * k / nshards); };
  const uint32_t np = plan->n_pool, ns = plan->n_big - plan->n_pool;
  const uint32_t p0 = part(np, shard), p1 = part(np, shard + 1);
  const uint32_t b0 = np + part(ns, shard), b1 = np + part(ns, shard + 1);
  const uint32_t m0 = part(plan->n_mid, shard), m1 = part(plan->n_mid, shard + 1);
  const uint32_t w0 = part(plan->n_light, shard), w1 = part(plan->n_light, shard + 1);
  auto big = k_k4_cta<kK4BigThreads, kK4BigLog, kK4BigRowWords>;
  auto pool = k_k4_pool;
  const size_t smem_pool = 2 * (1u << kK4PoolLog) * 4;
  auto mid = k_k4_cta<kK4MidThreads, kK4MidLog, kK4MidRowWords>;
  const size_t smem_big = (2 * (1u << kK4BigLog) + kK4BigRowWords) * 4;
  const size_t smem_mid = (2 * (1u << kK4MidLog) + kK4MidRowWords) * 4;
  const size_t smem_warp = (size_t)kK4WarpCtaWarps * kK4WarpWords * 4;
  static bool attr[64] = {false};
  const int dev = device_ordinal();
  if (dev < 64 && !attr[dev]) {
    GARY_CUDA(cudaFuncSetAttribute(big, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_big));
    GARY_CUDA(cudaFuncSetAttribute(pool, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_pool));
    GARY_CUDA(cudaFuncSetAttribute(mid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_mid));
    GARY_CUDA(cudaFuncSetAttribute(k_k4_warp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_warp));
    attr[dev] = true;
  }
  int per_mid = 0, per_warp = 0, per_pool = 0, per_big = 0;
  GARY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_big, big, kK4BigThreads, smem_big));
  per_big = std::max(per_big, 1);
  GARY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_pool, pool, kK4BigThreads, smem_pool));
  per_pool = std::max(per_pool, 1);
  GARY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_mid, mid, kK4MidThreads, smem_mid));
  GARY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_warp, k_k4_warp, kK4WarpCtaWarps * 32,
                                                          smem_warp));
  per_mid = std::max(per_mid, 1);
  per_warp = std::max(per_warp, 1);
  const uint64_t dmax = plan->max_pre;
  const uint64_t pool_words = plan->cursors.p ? dmax * ((dmax + 31) / 32) : 0;
  SchedState *st = plan->sched.p;
  GARY_CUDA(cudaMemsetAsync(st, 0, sizeof(SchedState), s));
  GARY_CUDA(cudaMemsetAsync(d_out, 0, 8, s));
  GARY_CUDA(cudaEventRecord(g->ev0, s));
  const GraphView gv = g->view();
  // The HBM-row vertices are the largest: their kernel runs first.
  if (p1 > p0) {
    // rows in HBM: the pool holds one row buffer per CTA of the grid
    const unsigned grid = std::min<unsigned>({(unsigned)(sm_count() * per_pool), plan->win_ctas, p1 - p0});
    if (!plan->cursors.p) {
      set_error("4-clique row pool missing for %u vertices", p1 - p0);
      return GARY_ERR_INVALID;
    }
    pool<<<grid, kK4BigThreads, smem_pool, s>>>(gv, plan->big.p, p0, p1, plan->cursors.p, pool_words,
                                                &st->next_cta, &st->error, d_out);
  }
  if (b1 > b0)  // rows in shared memory, two CTAs per SM
    big<<<std::min<unsigned>((unsigned)(sm_count() * per_big), b1 - b0), kK4BigThreads, smem_big, s>>>(
        gv, plan->big.p, b0, b1, nullptr, 0, &st->next_big, &st->error, d_out);
  if (m1 > m0)
    mid<<<std::min<unsigned>((unsigned)(sm_count() * per_mid), m1 - m0), kK4MidThreads, smem_mid, s>>>(
        gv, plan->mid.p, m0, m1, nullptr, 0, &st->next_aux, &st->error, d_out);
  if (w1 > w0)
    k_k4_warp<<<(unsigned)(sm_count() * per_warp), kK4WarpCtaWarps * 32, smem_warp, s>>>(
        gv, plan->light.p, w0, w1, &st->next_warp, &st->error, d_out);
  GARY_CUDA(cudaGetLastError());
  GARY_CUDA(cudaEventRecord(g->ev1, s));
  g->last = gary_count_stats{};
  g->last.tiles = (p1 - p0) + (b1 - b0) + (m1 - m0) + (w1 - w0);
  g->last.cta_tiles = (p1 - p0) + (b1 - b0) + (m1 - m0);
  g->last_timed = true;
  g->last_sched = st;
  g->last_span = nullptr;
  return GARY_OK;
}

int build_c4_plan(gary_graph *g, cudaStream_t s, PatternPlan **out) {
  GARY_TRY(build_symmetric(g, s));
  auto plan = std::make_unique<PatternPlan>();
  const uint32_t n = g->n;
  ScratchAlloc pol_alloc{s};
  auto pol = thrust::cuda::par_nosync(pol_alloc).on(s);
  DevBuf<uint8_t> cls;
  GARY_TRY(cls.alloc(n, s));
  k_c4_classify<<<grid_for(n), kThreads, 0, s>>>(g->sym.row.p, g->sym.adj.p, g->dag.outdeg.p, n,
                                                 (uint32_t)kC4LightWedges, cls.p);
  GARY_CUDA(cudaGetLastError());
  GARY_TRY(plan->light.alloc_persistent(std::max<uint32_t>(n, 1)));
  plan->n_light = (uint32_t)(thrust::copy_if(pol, thrust::counting_iterator<uint32_t>(0),
                                             thrust::counting_iterator<uint32_t>(n), plan->light.p,
                                             ClassIs{cls.p, kClassLight}) - plan->light.p);
  // the rest: exact wedge counts, then medium (a CTA hash map) or heavy (windows)
  DevBuf<uint32_t> big;
  GARY_TRY(big.alloc(std::max<uint32_t>(n, 1), s));
  const uint32_t nb = (uint32_t)(thrust::copy_if(pol, thrust::counting_iterator<uint32_t>(0),
                                                 thrust::counting_iterator<uint32_t>(n), big.p,
                                                 ClassIs{cls.p, kClassCta}) - big.p);
  DevBuf<uint64_t> wed;
  GARY_TRY(wed.alloc(std::max<uint32_t>(nb, 1), s));
  if (nb) {
    k_c4_exact_wedges<<<grid_for((uint64_t)nb * 32), kThreads, 0, s>>>(g->sym.row.p, g->sym.adj.p,
                                                                       g->dag.outdeg.p, big.p, nb, wed.p);
    GARY_CUDA(cudaGetLastError());
  }
  GARY_TRY(plan->mid.alloc_persistent(std::max<uint32_t>(nb, 1)));
  plan->n_mid = (uint32_t)(thrust::copy_if(pol, big.p, big.p + nb, wed.p, plan->mid.p,
                                           AtMost{kMidWedges}) - plan->mid.p);
  DevBuf<uint32_t> heavy;
  DevBuf<uint64_t> cost;
  GARY_TRY(heavy.alloc(std::max<uint32_t>(nb, 1), s));
  const uint32_t nh = (uint32_t)(thrust::copy_if(pol, big.p, big.p + nb, wed.p, heavy.p,
                                                 Above{kMidWedges}) - heavy.p);
  GARY_TRY(cost.alloc(std::max<uint32_t>(nh, 1), s));
  GARY_TRY(c4_win_attr());
  {
    int per_sm = 0;
    GARY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_c4_win, kWinThreads,
                                                            (size_t)kWinWords * 4));
    plan->win_ctas = (uint32_t)(sm_count() * std::max(per_sm, 1));
  }
  if (nh) {
    DevBuf<uint64_t> hw;
    GARY_TRY(hw.alloc(nh, s));
    thrust::copy_if(pol, wed.p, wed.p + nb, wed.p, hw.p, Above{kMidWedges});
    k_c4_heavy_cost<<<grid_for(nh), kThreads, 0, s>>>(g->sym.row.p, g->dag.outdeg.p, heavy.p, hw.p,
                                                      nh, cost.p);
    GARY_CUDA(cudaGetLastError());
    // biggest vertices first; tiles of about 1/8 of a CTA's share of the work
    thrust::sort_by_key(pol, cost.p, cost.p + nh, heavy.p, thrust::greater<uint64_t>());
    const uint64_t total = thrust::reduce(pol, cost.p, cost.p + nh, 0ull);
    const uint64_t target = std::max<uint64_t>(total / ((uint64_t)plan->win_ctas * 8), 1ull << 22);
    DevBuf<uint32_t> kt;
    GARY_TRY(kt.alloc((uint64_t)nh + 1, s));
    k_c4_tile_counts<<<grid_for(nh), kThreads, 0, s>>>(heavy.p, cost.p, nh, target, kt.p);
    GARY_CUDA(cudaMemsetAsync(kt.p + nh, 0, 4, s));
    thrust::exclusive_scan(pol, kt.p, kt.p + nh + 1, kt.p, 0u);
    uint32_t nt = 0;
    GARY_CUDA(cudaMemcpyAsync(&nt, kt.p + nh, 4, cudaMemcpyDeviceToHost, s));
    plan->max_pre = thrust::transform_reduce(pol, heavy.p, heavy.p + nh,
                                             PreOf{g->sym.row.p, g->dag.outdeg.p}, 0u, MaxU32());
    GARY_CUDA(cudaStreamSynchronize(s));
    plan->n_cta = nt;
    GARY_TRY(plan->tiles.alloc_persistent(std::max<uint32_t>(nt, 1)));
    k_c4_fill_tiles<<<grid_for(nh), kThreads, 0, s>>>(g->sym.row.p, g->dag.outdeg.p, heavy.p, nh, kt.p,
                                                      plan->tiles.p);
    GARY_CUDA(cudaGetLastError());
    GARY_TRY(plan->cursors.alloc_persistent((uint64_t)plan->win_ctas * kC4ScratchWords *
                                            std::max(plan->max_pre, 1u)));
  }
  GARY_TRY(plan->sched.alloc_persistent(1));
  GARY_CUDA(cudaStreamSynchronize(s));
  *out = plan.release();
  return GARY_OK;
}

int launch_c4(gary_graph *g, PatternPlan *plan, unsigned long long *d_out, cudaStream_t s,
              uint32_t shard, uint32_t nshards) {
  // shards split the heavy tiles, the medium list and the light list
  auto part = [&](uint32_t total, uint32_t k) { return (uint32_t)((uint64_t)total * k / nshards); };
  const uint32_t t0 = part(plan->n_cta, shard), t1 = part(plan->n_cta, shard + 1);
  const uint32_t m0 = part(plan->n_mid, shard), m1 = part(plan->n_mid, shard + 1);
  const uint32_t l0 = part(plan->n_light, shard), l1 = part(plan->n_light, shard + 1);
  const size_t smem_small = (size_t)kPWarps * 2 * kPSlots * 4;
  const size_t smem_mid = (size_t)kMidWords * 4;
  const size_t smem_win = (size_t)kWinWords * 4;
  static bool attr[64] = {false};
  const int dev = device_ordinal();
  if (dev < 64 && !attr[dev]) {
    GARY_CUDA(cudaFuncSetAttribute(k_c4_small, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_small));
    GARY_CUDA(cudaFuncSetAttribute(k_c4_mid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_mid));
    attr[dev] = true;
  }
  GARY_TRY(c4_win_attr());
  int per_sm = 0;
  GARY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_c4_small, kPWarps * 32, smem_small));
  if (per_sm < 1) per_sm = 1;
  int per_sm_mid = 0;
  GARY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_mid, k_c4_mid, kMidThreads, smem_mid));
  if (per_sm_mid < 1) per_sm_mid = 1;
  const GraphView sv{g->n, g->sym.row.p, g->sym.adj.p, true};
  GARY_CUDA(cudaMemsetAsync(plan->sched.p, 0, sizeof(SchedState), s));
  GARY_CUDA(cudaMemsetAsync(d_out, 0, 8, s));
  GARY_CUDA(cudaEventRecord(g->ev0, s));
  if (t1 > t0)
    k_c4_win<<<std::min<uint32_t>(plan->win_ctas, t1 - t0), kWinThreads, smem_win, s>>>(
        sv, plan->tiles.p, t0, t1, plan->cursors.p, std::max(plan->max_pre, 1u), plan->sched.p, d_out);
  if (m1 > m0)
    k_c4_mid<<<std::min<uint32_t>((uint32_t)(sm_count() * per_sm_mid), m1 - m0), kMidThreads, smem_mid, s>>>(
        sv, g->dag.outdeg.p, plan->mid.p + m0, m1 - m0, plan->sched.p, d_out);
  if (l1 > l0)
    k_c4_small<<<(unsigned)(sm_count() * per_sm), kPWarps * 32, smem_small, s>>>(
        sv, g->dag.outdeg.p, plan->light.p + l0, l1 - l0, plan->sched.p, d_out);
  GARY_CUDA(cudaGetLastError());
  GARY_CUDA(cudaEventRecord(g->ev1, s));
  g->last = gary_count_stats{};
  g->last.tiles = (t1 - t0) + (m1 - m0) + (l1 - l0);
  g->last.cta_tiles = (t1 - t0) + (m1 - m0);
  g->last_timed = true;
  g->last_sched = plan->sched.p;
  g->last_span = nullptr;
  return GARY_OK;
}

}  // namespace gary
