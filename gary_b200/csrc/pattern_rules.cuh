// Capacity rules of the 4-cycle and 4-clique kernels: which worker takes a
// vertex, and the shared-memory tables and row buffers that worker brings.
// The plans (patterns.cu) classify vertices with these functions, the kernels
// size their tables from these constants, and the host-only program
// tests/cpp/capacity_test.cu checks, at every class boundary and on
// adversarial degree patterns, that no table can fill past half and no
// counter or row buffer can overflow.  Host and device code; no CUDA calls.
#pragma once
#include <cstdint>

namespace gary {

// ---- 4-cycles ---------------------------------------------------------------
// A light vertex's wedges w go to a warp's hash map of kC4WarpSlots slots.  The
// plan's bound on its wedge count (sum over lower neighbours v of d(v), at
// least the distinct w) keeps it at most half full.
constexpr uint32_t kC4WarpSlots = 1024;
constexpr uint64_t kC4LightWedges = kC4WarpSlots / 2;
// A medium vertex (exact wedge count at most kC4MidWedges) gets a CTA map of
// kC4MidSlots slots with 16-bit counts: a count c(u, w) never exceeds the
// vertex's wedge count, since each v adds at most one to it.
constexpr uint32_t kC4MidSlots = 16384;
constexpr uint64_t kC4MidWedges = kC4MidSlots / 2;
// Heavy vertices count in windows: 16-bit counters while c(u, w) <= the
// number of lower neighbours fits, 32-bit ones (half windows) beyond.
constexpr uint32_t kC4Win16MaxPre = 0xFFFFu;

enum C4Class : uint8_t { kC4None = 0, kC4Light = 1, kC4Mid = 2, kC4Heavy = 3 };

// `bound`: the plan's upper bound of the wedge count; `exact`: the exact count
// (needed only when the bound rules out a light vertex).
__host__ __device__ constexpr C4Class c4_class(uint32_t pre, uint64_t bound, uint64_t exact) {
  return pre == 0 ? kC4None : bound <= kC4LightWedges ? kC4Light : exact <= kC4MidWedges ? kC4Mid : kC4Heavy;
}

__host__ __device__ constexpr bool c4_wide_counters(uint32_t pre) { return pre > kC4Win16MaxPre; }

// ---- 4-cliques --------------------------------------------------------------
// Largest d+(u) the 4-clique kernels take (the API refuses larger graphs).
constexpr uint32_t kK4MaxOutDegree = 4096;
constexpr uint32_t kK4WarpMaxD = 128;  // one warp per vertex up to here
constexpr uint32_t kK4MidMaxD = 362;   // a 256-thread CTA up to here, a 1024-thread CTA beyond
constexpr int kK4WarpLog = 8;          // position hash slots (log2) of each worker
constexpr int kK4MidLog = 10;
constexpr int kK4BigLog = 11;          // shared-row vertices: d+ <= 877
constexpr int kK4PoolLog = 13;         // HBM-row vertices: d+ <= 4096
// Shared words for bit rows: a warp's region, the 256-thread CTA's, the
// 1024-thread CTA's (96 KiB, so that two CTAs share an SM).  Past the last,
// rows live in an HBM buffer per CTA.
constexpr uint32_t kK4WarpRowWords = kK4WarpMaxD * ((kK4WarpMaxD + 31) / 32);  // 512
constexpr uint32_t kK4MidRowWords = kK4MidMaxD * ((kK4MidMaxD + 31) / 32);
constexpr uint32_t kK4BigRowWords = 24576;

enum K4Worker : uint8_t { kK4None = 0, kK4Warp = 1, kK4Mid = 2, kK4Big = 3, kK4Pool = 4 };

// Words of one bit row of a d-vertex subgraph.
__host__ __device__ constexpr uint32_t k4_row_words(uint32_t d) { return (d + 31) >> 5; }

// Vertices with fewer than 3 higher neighbours have no 4-clique.
__host__ __device__ constexpr K4Worker k4_worker(uint32_t d) {
  return d < 3 ? kK4None
         : d <= kK4WarpMaxD ? kK4Warp
         : d <= kK4MidMaxD ? kK4Mid
         : (uint64_t)d * k4_row_words(d) <= kK4BigRowWords ? kK4Big
                                                            : kK4Pool;
}

__host__ __device__ constexpr int k4_table_log(K4Worker w) {
  return w == kK4Warp ? kK4WarpLog : w == kK4Mid ? kK4MidLog : w == kK4Big ? kK4BigLog : kK4PoolLog;
}

// Shared row words of a worker (0: rows in its HBM buffer).
__host__ __device__ constexpr uint32_t k4_shared_row_words(K4Worker w) {
  return w == kK4Warp ? kK4WarpRowWords : w == kK4Mid ? kK4MidRowWords : w == kK4Big ? kK4BigRowWords : 0u;
}

// log2 of the position table a vertex asks for: at least 2d slots and 32
// (the kernels' hash_log2), before the worker's table caps it.
__host__ __device__ constexpr int k4_wanted_log(uint32_t d) {
  int l = 5;
  while (l < 32 && (1ull << l) < 2ull * d) ++l;
  return l;
}

}  // namespace gary
