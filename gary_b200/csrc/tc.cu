// Triangle counting on the degree-oriented DAG (pattern K3).
//
// Reference: graph_query::triangleCountHom (include/kernels/GraphQueryHom.cuh:15-43)
// launches one warp per oriented COO edge and intersects N+(src) and N+(dst)
// by per-key binary search.  The count is the same number,
//     T = sum over (u,v) in E+ of |N+(u) & N+(v)|,
// computed here vertex-tile by vertex-tile:
//
//   tile (u, j0, j1): the warp (or CTA) builds a shared-memory set of N+(u)
//   once, then streams the lists N+(v) for v = N+(u)[j], j0 <= j < j1, with
//   all 32 lanes busy, and counts members.  N+(u) is read once per tile
//   instead of once per edge; every N+(v) read is a coalesced sweep.
//
// Work is cut into weighted tiles (cost ~ wedges d+(v) + set build) and
// handed out by a persistent scheduler (sched.cuh): CTA tiles for vertices
// whose list does not fit a warp's table, then warp tiles.
#include <thrust/binary_search.h>
#include <thrust/execution_policy.h>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/transform_iterator.h>
#include <thrust/scan.h>
#include <thrust/transform.h>

#include <algorithm>
#include <exception>
#include <new>

#include "bulk.cuh"
#include "graph.cuh"
#include "tc.cuh"
#include "warp_ops.cuh"

namespace gary {

// ---------------------------------------------------------------------------
// Tile plan
namespace {

constexpr int kThreads = 256;

inline unsigned grid_for(uint64_t items) {
  uint64_t b = (items + kThreads - 1) / kThreads;
  uint64_t cap = (uint64_t)sm_count() * 16;
  return (unsigned)std::max<uint64_t>(std::min(b, cap), 1);
}

__host__ __device__ __forceinline__ uint64_t min_u64(uint64_t a, uint64_t b) { return a < b ? a : b; }

// per-vertex classification for the plain plan
__global__ void k_classify(const uint2 *__restrict__ row, const uint64_t *__restrict__ wedge,
                           uint32_t n, PlanParams pp, uint8_t *__restrict__ vclass,
                           uint64_t *__restrict__ costL, uint32_t *__restrict__ kW,
                           uint32_t *__restrict__ kC) {
  for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n;
       u += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t du = row[u].y;
    uint8_t cls = kClassNone;
    uint64_t cl = 0;
    uint32_t kw = 0, kc = 0;
    if (du >= 2) {
      const uint64_t c = wedge[u] + du + pp.vertex_overhead;
      if (du > pp.warp_cap) {
        cls = kClassCta;
        kc = (uint32_t)min_u64((c + pp.cta_tile_cost - 1) / pp.cta_tile_cost, du - 1);
      } else if (c > pp.warp_tile_cost) {
        cls = kClassSplit;
        kw = (uint32_t)min_u64((c + pp.warp_tile_cost - 1) / pp.warp_tile_cost, du - 1);
      } else {
        cls = kClassLight;
        cl = c;
      }
    }
    vclass[u] = cls;
    costL[u] = cl;
    kW[u] = kw;
    kC[u] = kc;
  }
}

__global__ void k_fill_split_tiles(const uint2 *__restrict__ row, uint32_t n,
                                   const uint32_t *__restrict__ k, const uint32_t *__restrict__ off,
                                   Tile *__restrict__ tiles) {
  for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u < n;
       u += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t kk = k[u];
    if (!kk) continue;
    // the last neighbour never closes a triangle as the middle vertex
    const uint32_t span = row[u].y - 1;
    const uint32_t o = off[u];
    for (uint32_t i = 0; i < kk; ++i) {
      Tile t;
      t.u0 = (uint32_t)u;
      t.u1 = (uint32_t)u + 1;
      t.j0 = (uint32_t)((uint64_t)i * span / kk);
      t.j1 = (uint32_t)((uint64_t)(i + 1) * span / kk);
      tiles[o + i] = t;
    }
  }
}

struct GroupTarget {
  uint64_t tw;
  __host__ __device__ uint64_t operator()(uint64_t g) const { return g * tw; }
};

__global__ void k_fill_group_tiles(const uint32_t *__restrict__ starts, uint64_t G, uint32_t n,
                                   Tile *__restrict__ tiles) {
  for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < G;
       g += (uint64_t)gridDim.x * blockDim.x) {
    Tile t;
    t.u0 = starts[g];
    t.u1 = g + 1 < G ? starts[g + 1] : n;
    t.j0 = 0;
    t.j1 = kGroupTile;
    tiles[g] = t;
  }
}

}  // namespace

int build_plain_plan(gary_graph *g, const PlanParams &pp, cudaStream_t s, gary_count_plan **out) {
  auto plan = std::make_unique<gary_count_plan>();
  plan->params = pp;
  const uint32_t n = g->n;
  auto pol = thrust::cuda::par_nosync.on(s);
  GARY_TRY(plan->vclass.alloc_persistent(n));
  DevBuf<uint64_t> costL;
  DevBuf<uint32_t> kW, kC;
  GARY_TRY(costL.alloc((uint64_t)n + 1, s));
  GARY_TRY(kW.alloc((uint64_t)n + 1, s));
  GARY_TRY(kC.alloc((uint64_t)n + 1, s));
  k_classify<<<grid_for(n), kThreads, 0, s>>>(g->row.p, g->wedge.p, n, pp, plan->vclass.p, costL.p,
                                              kW.p, kC.p);
  GARY_CUDA(cudaGetLastError());
  GARY_CUDA(cudaMemsetAsync(costL.p + n, 0, 8, s));
  GARY_CUDA(cudaMemsetAsync(kW.p + n, 0, 4, s));
  GARY_CUDA(cudaMemsetAsync(kC.p + n, 0, 4, s));
  thrust::exclusive_scan(pol, costL.p, costL.p + n + 1, costL.p, 0ull);
  thrust::exclusive_scan(pol, kW.p, kW.p + n + 1, kW.p, 0u);
  thrust::exclusive_scan(pol, kC.p, kC.p + n + 1, kC.p, 0u);
  uint64_t totalL = 0;
  uint32_t nW = 0, nC = 0;
  GARY_CUDA(cudaMemcpyAsync(&totalL, costL.p + n, 8, cudaMemcpyDeviceToHost, s));
  GARY_CUDA(cudaMemcpyAsync(&nW, kW.p + n, 4, cudaMemcpyDeviceToHost, s));
  GARY_CUDA(cudaMemcpyAsync(&nC, kC.p + n, 4, cudaMemcpyDeviceToHost, s));
  GARY_CUDA(cudaStreamSynchronize(s));
  const uint64_t G = totalL ? (totalL + pp.warp_tile_cost - 1) / pp.warp_tile_cost : 0;
  const uint64_t total = (uint64_t)nC + nW + G;
  if (total >= (1ull << 31)) {
    set_error("tile plan too large (%llu tiles)", (unsigned long long)total);
    return GARY_ERR_UNSUPPORTED;
  }
  plan->n_cta = nC;
  plan->n_warp = (uint32_t)(nW + G);
  GARY_TRY(plan->tiles.alloc_persistent(std::max<uint64_t>(total, 1)));
  // the row length array is needed by the split-tile fill; kW/kC hold offsets
  // after the scans, and the per-vertex counts are offsets' differences, so
  // recompute counts from the classification directly.
  {
    DevBuf<uint32_t> cntW, cntC;
    GARY_TRY(cntW.alloc(n, s));
    GARY_TRY(cntC.alloc(n, s));
    thrust::transform(pol, kW.p + 1, kW.p + n + 1, kW.p, cntW.p, thrust::minus<uint32_t>());
    thrust::transform(pol, kC.p + 1, kC.p + n + 1, kC.p, cntC.p, thrust::minus<uint32_t>());
    k_fill_split_tiles<<<grid_for(n), kThreads, 0, s>>>(g->row.p, n, cntC.p, kC.p, plan->tiles.p);
    k_fill_split_tiles<<<grid_for(n), kThreads, 0, s>>>(g->row.p, n, cntW.p, kW.p,
                                                       plan->tiles.p + nC);
    GARY_CUDA(cudaGetLastError());
  }
  if (G) {
    DevBuf<uint32_t> starts;
    GARY_TRY(starts.alloc(G, s));
    auto targets = thrust::make_transform_iterator(thrust::counting_iterator<uint64_t>(0),
                                                   GroupTarget{pp.warp_tile_cost});
    thrust::lower_bound(pol, costL.p, costL.p + n, targets, targets + G, starts.p);
    k_fill_group_tiles<<<grid_for(G), kThreads, 0, s>>>(starts.p, G, n,
                                                       plan->tiles.p + nC + nW);
    GARY_CUDA(cudaGetLastError());
  }
  GARY_TRY(plan->sched.alloc_persistent(1));
  GARY_TRY(plan->result.alloc_persistent(1));
  GARY_CUDA(cudaStreamSynchronize(s));
  *out = plan.release();
  return GARY_OK;
}

// ---------------------------------------------------------------------------
// Counting kernel
namespace {

template <int WARPS>
struct TcSmem {
  static constexpr uint32_t kWords = WARPS * kWarpTableSlots;
};

// CTA tile: u has more out-neighbours than a warp table holds.
//   d+(u) <= cta_slots/2 : CTA-wide hash set of N+(u)
//   otherwise            : N+(u) staged (TMA bulk) or sampled into shared
//                          memory, two-phase search per probe
template <int WARPS>
__device__ uint32_t cta_tile(const GraphView &g, const Tile &t, uint32_t *smem, uint64_t *bar,
                             uint32_t &phase, unsigned *err) {
  constexpr uint32_t S = WARPS * kWarpTableSlots;  // shared words
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint2 ru = g.row[t.u0];
  const uint32_t du = ru.y;
  const uint32_t *au = g.adj + (uint64_t)ru.x * 4;
  const uint32_t j0 = t.j0, j1 = min(t.j1, du - 1);
  uint32_t cnt = 0;
  if (j0 >= j1) return 0;
  const uint32_t keys_lo = j0 + 1;  // members of N+(u) that can close a triangle
  const uint32_t nkeys = du - keys_lo;
  if (nkeys * 2 <= S) {
    const int logT = hash_log2(nkeys);
    for (uint32_t i = threadIdx.x; i < (1u << logT); i += blockDim.x) smem[i] = kSentinel;
    __syncthreads();
    hash_insert_range(smem, logT, au, keys_lo, du, threadIdx.x, blockDim.x);
    __syncthreads();
    cnt = warp_walk_lists(g, au, j0 + warp * 32, j1, WARPS * 32, lane,
                          [&](uint32_t w) { return hash_contains(smem, logT, w); });
  } else {
    // stage the whole list when it fits, else keep S samples (two-phase)
    if (du <= S) {
      if (threadIdx.x == 0) bulk_stage(smem, au, ((du + 3) / 4) * 16, bar);
      __syncthreads();
      if (!mbar_wait_bounded(bar, phase)) {
        if (threadIdx.x == 0) atomicOr(err, 1u);
        mbar_wait_bounded(bar, phase);  // drain the copy before leaving
      }
      phase ^= 1;
    } else {
      for (uint32_t i = threadIdx.x; i < S; i += blockDim.x) smem[i] = au[(uint64_t)i * du / S];
      __syncthreads();
    }
    cnt = warp_walk_lists(g, au, j0 + warp * 32, j1, WARPS * 32, lane,
                          [&](uint32_t w) { return search_2phase(au, du, smem, S, w); });
  }
  // the next tile rewrites shared memory, possibly through the async proxy
  fence_proxy_async_smem();
  __syncthreads();
  return cnt;
}

// Warp tile on one vertex: hash N+(u)[j0+1..) in the warp's table, walk the lists.
__device__ __forceinline__ uint32_t warp_vertex(const GraphView &g, uint32_t u, uint32_t j0,
                                                uint32_t j1, uint32_t *tab, int lane) {
  const uint2 ru = g.row[u];
  const uint32_t du = ru.y;
  if (du < 2) return 0;
  j1 = min(j1, du - 1);
  if (j0 >= j1) return 0;
  const uint32_t *au = g.adj + (uint64_t)ru.x * 4;
  const int logT = hash_log2(du - j0 - 1);
  for (uint32_t i = lane; i < (1u << logT); i += 32) tab[i] = kSentinel;
  __syncwarp();
  hash_insert_range(tab, logT, au, j0 + 1, du, lane, 32);
  __syncwarp();
  uint32_t c = warp_walk_lists(g, au, j0, j1, 32, lane,
                               [&](uint32_t w) { return hash_contains(tab, logT, w); });
  __syncwarp();
  return c;
}

template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32, 2)
    k_tc_persistent(GraphView g, const uint8_t *__restrict__ vclass, const Tile *__restrict__ tiles,
                    uint32_t n_cta, uint32_t n_warp, TileRange rng, SchedState *sched,
                    unsigned long long *__restrict__ out) {
  extern __shared__ __align__(16) uint32_t smem[];
  __shared__ uint64_t bar;
  __shared__ uint32_t s_tile;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long cnt = 0;

  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_fence_init();
  }
  __syncthreads();
  uint32_t phase = 0;

  // phase 1: CTA tiles, largest work first by construction of the plan
  while (true) {
    if (threadIdx.x == 0) s_tile = rng.cta_lo + atomicAdd(&sched->next_cta, 1u);
    __syncthreads();
    const uint32_t t = s_tile;
    __syncthreads();
    if (t >= rng.cta_hi) break;
    const Tile tl = tiles[t];
    cnt += cta_tile<WARPS>(g, tl, smem, &bar, phase, &sched->error);
  }

  // phase 2: warp tiles, each warp on its own table
  uint32_t *tab = smem + warp * kWarpTableSlots;
  const Tile *wt = tiles + n_cta;
  while (true) {
    uint32_t t = 0;
    if (lane == 0) t = rng.warp_lo + atomicAdd(&sched->next_warp, 1u);
    t = __shfl_sync(kFull, t, 0);
    if (t >= rng.warp_hi) break;
    const Tile tl = wt[t];
    if (tl.j1 != kGroupTile) {
      cnt += warp_vertex(g, tl.u0, tl.j0, tl.j1, tab, lane);
      continue;
    }
    // a group of light vertices: take them 32 at a time
    for (uint32_t ub = tl.u0; ub < tl.u1; ub += 32) {
      const uint32_t uu = ub + lane;
      const bool light = uu < tl.u1 && vclass[uu] == kClassLight;
      unsigned m = __ballot_sync(kFull, light);
      while (m) {
        const int k = __ffs(m) - 1;
        m &= m - 1;
        cnt += warp_vertex(g, ub + k, 0, 0xFFFFFFFEu, tab, lane);
      }
    }
  }

  cnt = warp_sum_u64(cnt);
  if (lane == 0 && cnt) atomicAdd(out, cnt);
  if (threadIdx.x == 0) mbar_inval(&bar);
}

}  // namespace

int launch_plain_k3(gary_graph *g, gary_count_plan *plan, unsigned long long *d_out,
                    cudaStream_t s, uint32_t shard, uint32_t nshards) {
  constexpr int WARPS = kTcWarps;
  const size_t smem = (size_t)TcSmem<WARPS>::kWords * 4;
  static bool attr_done[64] = {false};
  int dev = device_ordinal();
  if (dev < 64 && !attr_done[dev]) {
    GARY_CUDA(cudaFuncSetAttribute(k_tc_persistent<WARPS>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr_done[dev] = true;
  }
  int per_sm = 0;
  GARY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tc_persistent<WARPS>,
                                                          WARPS * 32, smem));
  if (per_sm < 1) per_sm = 1;
  const unsigned grid = (unsigned)(sm_count() * per_sm);
  const TileRange rng = shard_range(plan->n_cta, plan->n_warp, shard, nshards);
  GARY_CUDA(cudaMemsetAsync(plan->sched.p, 0, sizeof(SchedState), s));
  GARY_CUDA(cudaMemsetAsync(d_out, 0, sizeof(unsigned long long), s));
  GARY_CUDA(cudaEventRecord(g->ev0, s));
  k_tc_persistent<WARPS><<<grid, WARPS * 32, smem, s>>>(g->view(), plan->vclass.p, plan->tiles.p,
                                                        plan->n_cta, plan->n_warp, rng,
                                                        plan->sched.p, d_out);
  GARY_CUDA(cudaGetLastError());
  GARY_CUDA(cudaEventRecord(g->ev1, s));
  g->last = gary_count_stats{};
  g->last.tiles = (rng.cta_hi - rng.cta_lo) + (rng.warp_hi - rng.warp_lo);
  g->last.cta_tiles = rng.cta_hi - rng.cta_lo;
  g->last_timed = true;
  return GARY_OK;
}

}  // namespace gary
