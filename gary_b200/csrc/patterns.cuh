// Plans and launches of the 4-clique and 4-cycle kernels (patterns.cu).
#pragma once
#include <cstdint>

#include "graph.cuh"
#include "pattern_rules.cuh"
#include "tc.cuh"

namespace gary {

struct PatternPlan {
  // K4: CTA tiles then warp tiles.  C4: window tiles of heavy vertices, as
  // {v0 = u, v1 = |N(u) below u|, j0 = first window, j1 = end window}.
  DevBuf<Tile> tiles;
  DevBuf<uint32_t> light;    // light vertices (K4 groups index it; C4 warps walk it)
  DevBuf<uint32_t> mid;      // C4: medium vertices, one CTA hash map each; K4: mid vertices
  DevBuf<uint32_t> big;      // K4: vertices with d+ > 512, largest first (the n_pool with rows in HBM first)
  DevBuf<uint32_t> cursors;  // C4: per window-kernel CTA, 6 x max_pre words of list state; K4: row pool
  DevBuf<SchedState> sched;
  uint32_t n_cta = 0, n_warp = 0, n_light = 0, n_mid = 0, n_big = 0, n_pool = 0, max_pre = 0, win_ctas = 0;
};

int build_k4_plan(gary_graph *g, cudaStream_t s, PatternPlan **out);
int launch_k4(gary_graph *g, PatternPlan *plan, unsigned long long *d_out, cudaStream_t s,
              uint32_t shard, uint32_t nshards);
int build_c4_plan(gary_graph *g, cudaStream_t s, PatternPlan **out);
int launch_c4(gary_graph *g, PatternPlan *plan, unsigned long long *d_out, cudaStream_t s,
              uint32_t shard, uint32_t nshards);

}  // namespace gary
