// Tile plans and launch entry points of the counting kernels.
#pragma once
#include <cstdint>

#include "graph.cuh"
#include "internal.cuh"

namespace gary {

constexpr int kTcWarps = 16;               // warps per CTA of the counting kernel
constexpr uint32_t kWarpTableSlots = 1024;  // per-warp shared hash table (4 KB)
constexpr uint32_t kGroupTile = 0xFFFFFFFFu;

enum : uint8_t { kClassNone = 0, kClassLight = 1, kClassSplit = 2, kClassCta = 3 };

// A unit of scheduled work.
//   j1 == kGroupTile : every light vertex u in [u0, u1), whole lists
//   otherwise        : vertex u0 only, middle vertices N+(u0)[j0..j1)
struct Tile {
  uint32_t u0, u1, j0, j1;
};

struct PlanParams {
  uint32_t warp_cap = kWarpTableSlots / 2;  // largest d+(u) a warp table takes
  uint64_t warp_tile_cost = 1u << 13;       // target work per warp tile
  uint64_t cta_tile_cost = 1u << 17;        // target work per CTA tile
  uint64_t vertex_overhead = 48;            // fixed cost of a vertex (row loads, table clear)
};

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
  uint32_t error;
  uint32_t pad;
};

}  // namespace gary

struct gary_count_plan {
  gary::PlanParams params;
  gary::DevBuf<uint8_t> vclass;
  gary::DevBuf<gary::Tile> tiles;
  uint32_t n_cta = 0;
  uint32_t n_warp = 0;
  gary::DevBuf<gary::SchedState> sched;
  gary::DevBuf<unsigned long long> result;
};

namespace gary {
int build_plain_plan(gary_graph *g, const PlanParams &pp, cudaStream_t s, gary_count_plan **out);
int launch_plain_k3(gary_graph *g, gary_count_plan *plan, unsigned long long *d_out,
                    cudaStream_t s, uint32_t shard, uint32_t nshards);
}  // namespace gary
