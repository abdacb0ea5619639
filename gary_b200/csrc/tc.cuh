// Tile plans and launch entry points of the counting kernels.
#pragma once
#include <cstdint>

#include "bulk.cuh"
#include "graph.cuh"
#include "internal.cuh"

namespace gary {

// Warps per CTA of the counting kernel at `min_blocks` CTAs per SM: 16 at 2;
// 12 at 3, where 36 resident warps at 56 registers beat 48 warps held to 40
// registers with spills (RMAT-24 ef32 122.7 -> 119.7 ms, RMAT-22 7.05 -> 6.77 ms).
constexpr int tc_warps(int min_blocks) { return min_blocks >= 3 ? 12 : 16; }
constexpr int kTcMaxWarps = 16;
constexpr uint32_t kWarpTableSlots = 1024;  // per-warp shared set (4 KB)
constexpr uint32_t kGroupTile = 0xFFFFFFFFu;
constexpr uint32_t kMaxCountCtas = 1024;  // CTAs of a counting launch (SMs x resident CTAs)

enum : uint8_t { kClassNone = 0, kClassLight = 1, kClassSplit = 2, kClassCta = 3 };

// Intersection variants a tile can run (the cost model's output order).
enum : uint32_t { kVarHash = 0, kVarSearch = 1, kVarRegs = 2, kVarBitmap = 3 };

// Can a warp run middle vertex v (d = d+(v), span = id span of N+(v)) with
// variant `var`?  Sizes follow the warp's kWarpTableSlots shared words.
__host__ __device__ __forceinline__ bool variant_legal(uint32_t var, uint32_t d, uint32_t span) {
  switch (var) {
    case kVarHash: return d <= kWarpTableSlots / 2;
    case kVarSearch: return d <= kWarpTableSlots;
    case kVarRegs: return d <= 8;
    case kVarBitmap: return span <= (kWarpTableSlots - 1) * 32u - 1u;
    default: return false;
  }
}

// A unit of scheduled work over middle vertices v.
//   j1 == kGroupTile : light vertices light[v0 .. v1) (the plan's compacted
//                      list of light vertices), all their in-edges
//   otherwise        : vertex v0 only, in-edges [j0, j1) of its in-list
struct Tile {
  uint32_t v0, v1, j0, j1;
};

// warp_tile_cost and min_blocks left at 0 follow the graph's total work
// (resolve_params): about 32 warp tiles per resident warp, and 3 resident CTAs
// per SM once there are 2^31 probes or more.
//
// cta_set_words and stage_polls change no plan, only how CTA tiles run; they
// exist so that tests can reach every CTA set path on small graphs:
// cta_set_words caps the shared words a CTA tile's set of N+(v) may use (the
// path is then chosen as if the CTA had only that much shared memory), and
// stage_polls caps the polls of the first wait for a bulk staging copy (the
// drain wait after a timeout always keeps the full limit).
struct PlanParams {
  uint32_t warp_cap = kWarpTableSlots / 2;  // largest d+(v) a warp set takes
  uint64_t warp_tile_cost = 0;              // target probes per warp tile (0: from the work)
  uint64_t cta_tile_cost = 1u << 20;        // target probes per CTA tile
  uint64_t vertex_overhead = 64;            // fixed cost of a middle vertex
  uint32_t min_blocks = 0;                  // resident CTAs per SM, 2 or 3 (0: from the work)
  uint32_t cta_set_words = 0;               // 0: the CTA's whole shared buffer
  uint32_t stage_polls = kSpinLimit;        // polls of the first staging wait
};

// The parameters a plan over `total_work` probes uses: explicit values as
// given, the zeros resolved.
PlanParams resolve_params(PlanParams pp, uint64_t total_work);

// Process-wide tuning overrides (0 = keep the default), set by gary_tune().
PlanParams tuned_params();

// Contiguous tile ranges of one shard (multi-GPU: every rank holds the whole
// graph and counts its own ranges; the partial counts are summed).
struct TileRange {
  uint32_t cta_lo, cta_hi, warp_lo, warp_hi;
};

inline TileRange shard_range(uint32_t n_cta, uint32_t n_warp, uint32_t shard, uint32_t nshards) {
  TileRange r;
  r.cta_lo = (uint32_t)((uint64_t)n_cta * shard / nshards);
  r.cta_hi = (uint32_t)((uint64_t)n_cta * (shard + 1) / nshards);
  r.warp_lo = (uint32_t)((uint64_t)n_warp * shard / nshards);
  r.warp_hi = (uint32_t)((uint64_t)n_warp * (shard + 1) / nshards);
  return r;
}

// Scheduler words, zeroed before every launch.
struct SchedState {
  uint32_t next_cta;
  uint32_t next_warp;
  uint32_t error;     // kLaunchErr* bits
  uint32_t next_aux;  // a third queue (the 4-cycle kernel's medium vertices)
  uint32_t cta_path[4];  // triangle CTA tiles by the set that held N+(v) (kPath*)
  uint32_t next_big;     // a fourth queue (4-clique vertices whose rows fit shared memory)
};

// Sets a triangle CTA tile can hold N+(v) in, cheapest first.
enum : uint32_t { kPathBitmap = 0, kPathBuckets = 1, kPathStaged = 2, kPathSampled = 3 };

// In-edge index of the middle-vertex formulation.  For every oriented edge
// u -> v whose list suffix after v is non-empty, and with d+(v) > 0:
//   inedge[k] = {first word of N+(u) after v, length of that suffix}
// grouped by v: v's records are inedge[inptr[v] .. inptr[v+1]).
struct InIndex {
  DevBuf<uint2> inedge;
  DevBuf<uint64_t> inptr;
  DevBuf<uint64_t> work;  // per v: sum of suffix lengths (probes)
  uint64_t records = 0;
  uint64_t total_work = 0;
};

}  // namespace gary

struct gary_count_plan {
  gary::PlanParams params;
  gary::InIndex in;
  gary::DevBuf<uint8_t> vclass;
  gary::DevBuf<uint32_t> light;  // light vertices (group tiles index this list)
  uint32_t n_light = 0;
  gary::DevBuf<gary::Tile> tiles;
  uint32_t n_cta = 0;
  uint32_t n_warp = 0;
  gary::DevBuf<gary::SchedState> sched;
  gary::DevBuf<uint8_t> variant;  // learned plans: intersection variant per middle vertex
  bool learned = false;
  // per CTA of the last launch: start and finish time (%globaltimer ns)
  gary::DevBuf<unsigned long long> span;
};

namespace gary {
// model: host copy of a cost-model parameter block (learned plan) or null
int build_k3_plan(gary_graph *g, const PlanParams &pp, cudaStream_t s, gary_count_plan **out,
                  const float *model = nullptr);
// Cost-model features and legal-variant masks of every middle vertex.
int k3_features(gary_graph *g, gary_count_plan *plan, float *d_x, uint8_t *d_legal, cudaStream_t s);
int launch_k3(gary_graph *g, gary_count_plan *plan, unsigned long long *d_out, cudaStream_t s,
              uint32_t shard, uint32_t nshards);
// The same launch with a forced per-vertex variant array and/or a per-vertex
// cycle log (profiling for the cost model).
int launch_k3_ctl(gary_graph *g, gary_count_plan *plan, unsigned long long *d_out, cudaStream_t s,
                  uint32_t shard, uint32_t nshards, const uint8_t *variant,
                  unsigned long long *cycles, unsigned long long *gcount = nullptr);
}  // namespace gary
