// Triangle counting on the degree-oriented DAG (pattern K3).
//
// Reference: graph_query::triangleCountHom (include/kernels/GraphQueryHom.cuh:15-43)
// launches one warp per oriented COO edge (u,v) and counts |N+(u) & N+(v)| by
// per-key binary search, one key per lane.  The total is the same number
//     T = sum over (u,v) in E+ of |N+(u) & N+(v)|,
// computed here from the MIDDLE vertex of each triangle u < v < w (ids are
// degree ranks, so every list is sorted in orientation order):
//
//     T = sum over v of  sum over in-edges u->v of |S(u,v) & N+(v)|,
//     S(u,v) = the part of N+(u) after v.
//
// One warp (or CTA) holds N+(v) as a shared-memory bitmap (when its id range
// is short) or hash set, and streams the suffixes S(u,v) of all in-edges of v
// with 16-byte loads over the padded lists, all lanes busy.  The probe count
// is sum over u of C(d+(u), 2), 3.5-4x fewer than streaming N+(v) for every
// edge (sum of d+(v)) on RMAT graphs, and every read is a coalesced sweep.
//
// Work is cut into tiles of bounded probe count over the in-edge index and
// served by a persistent scheduler: CTA tiles (large N+(v)) first, then warp
// tiles.
#include <cub/cub.cuh>
#include <thrust/binary_search.h>
#include <thrust/copy.h>
#include <thrust/execution_policy.h>
#include <thrust/fill.h>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/reverse_iterator.h>
#include <thrust/iterator/transform_iterator.h>
#include <thrust/reduce.h>
#include <thrust/scan.h>
#include <thrust/transform.h>

#include <algorithm>
#include <memory>

#include "bulk.cuh"
#include "mlp.cuh"
#include "graph.cuh"
#include "tc.cuh"
#include "warp_ops.cuh"

namespace gary {

// ---------------------------------------------------------------------------
// Plan: in-edge index + tiles
namespace {

constexpr int kThreads = 256;

inline unsigned grid_for(uint64_t items) {
  uint64_t b = (items + kThreads - 1) / kThreads;
  uint64_t cap = (uint64_t)sm_count() * 16;
  return (unsigned)std::max<uint64_t>(std::min(b, cap), 1);
}

inline int bits_for(uint64_t x) {
  int b = 0;
  while (b < 64 && (x - 1) >> b) ++b;
  return std::max(b, 1);
}

__host__ __device__ __forceinline__ uint64_t min_u64(uint64_t a, uint64_t b) { return a < b ? a : b; }

struct MinU64 {
  __host__ __device__ uint64_t operator()(uint64_t a, uint64_t b) const { return a < b ? a : b; }
};

// One candidate per padded word w of N+(u): the suffix after v = adj[w].
// Words without a record get the key n - 1: in rank ids the top vertex has
// no higher neighbour, so no record ever targets it, and the keys of an
// n = 2^k graph fit k bits (one radix pass fewer than with the key n).
__global__ void k_in_candidates(const uint2 *__restrict__ row, const uint32_t *__restrict__ adj,
                                const uint32_t *__restrict__ rowid, uint64_t words, uint32_t n,
                                uint32_t *__restrict__ keys, uint2 *__restrict__ vals) {
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < words;
       w += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t u = rowid[w];
    const uint2 r = row[u];
    const uint64_t pos = w - (uint64_t)r.x * 4;
    uint32_t key = n - 1;
    uint2 val = make_uint2(0, 0);
    if (pos < r.y) {
      const uint32_t v = adj[w];
      const uint32_t rem = r.y - (uint32_t)pos - 1;
      if (rem && row[v].y) {
        key = v;
        val = make_uint2((uint32_t)(w + 1), rem);
      }
    }
    keys[w] = key;
    vals[w] = val;
  }
}

// first index i with keys[i] >= x in a sorted array (one thread)
__global__ void k_first_geq(const uint32_t *__restrict__ keys, uint64_t len, uint32_t x,
                            uint64_t *__restrict__ out) {
  uint64_t b = 0, e = len;
  while (b < e) {
    const uint64_t m = (b + e) >> 1;
    if (keys[m] < x) b = m + 1;
    else e = m;
  }
  *out = b;
}

__global__ void k_in_heads(const uint32_t *__restrict__ keys, uint64_t m,
                           uint64_t *__restrict__ inptr) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = keys[i];
    if (i == 0 || keys[i - 1] != v) inptr[v] = i;
  }
}

// work[v] = sum of suffix lengths of v's in-edges (segmented warp scan; keys sorted).
__global__ void k_in_work(const uint32_t *__restrict__ keys, const uint2 *__restrict__ vals,
                          uint64_t m, unsigned long long *__restrict__ work) {
  const int lane = threadIdx.x & 31;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x; base < m; base += stride) {
    const uint64_t i = base + threadIdx.x;
    const bool ok = i < m;
    const uint32_t v = ok ? keys[i] : 0xFFFFFFFFu;
    unsigned long long x = ok ? vals[i].y : 0ull;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long t = __shfl_up_sync(kFull, x, o);
      const uint32_t tv = __shfl_up_sync(kFull, v, o);
      if (lane >= o && tv == v) x += t;
    }
    const uint32_t nv = __shfl_down_sync(kFull, v, 1);
    if (ok && (lane == 31 || nv != v) && x) atomicAdd(&work[v], x);
  }
}

// pcost (optional): predicted cycles of a warp-class vertex, with tile target
// tw_pred in the same unit; without it, costs are probe counts.
__global__ void k_classify(const uint2 *__restrict__ row, const uint32_t *__restrict__ adj,
                           const uint64_t *__restrict__ work,
                           const uint64_t *__restrict__ inptr, uint32_t n, PlanParams pp,
                           const uint64_t *__restrict__ pcost, uint64_t tw_pred,
                           uint8_t *__restrict__ vclass, uint64_t *__restrict__ costL,
                           uint32_t *__restrict__ kW, uint32_t *__restrict__ kC) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint2 rv = row[v];
    const uint32_t dv = rv.y;
    const uint64_t nin = inptr[v + 1] - inptr[v];
    uint8_t cls = kClassNone;
    uint64_t cl = 0;
    uint32_t kw = 0, kc = 0;
    if (dv && nin) {
      // a warp holds N+(v) as a bitmap when its id span is short, else as
      // buckets when d+(v) <= warp_cap; otherwise the CTA shares one set
      const uint32_t span = adj[(uint64_t)rv.x * 4 + dv - 1] - adj[(uint64_t)rv.x * 4];
      const bool bitmap = span <= bitmap_max_span(kWarpTableSlots);
      const bool warp_fits = bitmap || dv <= pp.warp_cap;
      const uint64_t build = bitmap ? (span >> 5) + dv : 4ull * dv;
      const bool pred = pcost && warp_fits;
      const uint64_t cp = work[v] + build + pp.vertex_overhead;  // probe cost
      // learned: predicted cycles, but never below the probe cost scaled to
      // the same tile target, so that no tile outgrows a plain one (a vertex
      // the model under-rates would otherwise end the launch alone)
      const uint64_t c = pred ? max(pcost[v] + 1, cp * tw_pred / pp.warp_tile_cost) : cp;
      const uint64_t tw = pred ? tw_pred : pp.warp_tile_cost;
      if (!warp_fits) {
        cls = kClassCta;
        kc = (uint32_t)min_u64((c + pp.cta_tile_cost - 1) / pp.cta_tile_cost, nin);
      } else if (c > tw) {
        cls = kClassSplit;
        kw = (uint32_t)min_u64((c + tw - 1) / tw, nin);
      } else {
        cls = kClassLight;
        cl = c;
      }
    }
    vclass[v] = cls;
    costL[v] = cl;
    kW[v] = kw;
    kC[v] = kc;
  }
}

// off[] holds exclusive tile offsets (n+1 entries): vertex v owns tiles
// off[v] .. off[v+1], splitting its in-edge list evenly.
__global__ void k_fill_split_tiles(const uint64_t *__restrict__ inptr, uint32_t n,
                                   const uint32_t *__restrict__ off, Tile *__restrict__ tiles) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t kk = off[v + 1] - off[v];
    if (!kk) continue;
    const uint64_t nin = inptr[v + 1] - inptr[v];
    const uint32_t o = off[v];
    for (uint32_t i = 0; i < kk; ++i) {
      Tile t;
      t.v0 = (uint32_t)v;
      t.v1 = (uint32_t)v + 1;
      t.j0 = (uint32_t)((uint64_t)i * nin / kk);
      t.j1 = (uint32_t)((uint64_t)(i + 1) * nin / kk);
      tiles[o + i] = t;
    }
  }
}

struct GroupTarget {
  uint64_t tw;
  __host__ __device__ uint64_t operator()(uint64_t g) const { return g * tw; }
};

struct IsLight {
  const uint8_t *vclass;
  __host__ __device__ bool operator()(uint32_t v) const { return vclass[v] == kClassLight; }
};

struct LightCost {
  const uint64_t *cost;
  __host__ __device__ uint64_t operator()(uint32_t v) const { return cost[v]; }
};

// Group tiles over the compacted light-vertex list: tile g covers list
// positions [starts[g], starts[g+1]).
__global__ void k_fill_group_tiles(const uint32_t *__restrict__ starts, uint64_t G, uint32_t L,
                                   Tile *__restrict__ tiles) {
  for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < G;
       g += (uint64_t)gridDim.x * blockDim.x) {
    Tile t;
    t.v0 = starts[g];
    t.v1 = g + 1 < G ? starts[g + 1] : L;
    t.j0 = 0;
    t.j1 = kGroupTile;
    tiles[g] = t;
  }
}

}  // namespace

// Cost-model features of middle vertex v (all log2(1 + .)):
//   x0 degree, x1 mean in-edge suffix length (the other endpoints' remaining
//   out-degree), x2 = x0 - x1 (their log ratio), x3 out-degree d+(v),
//   x4 id span of N+(v), x5 number of in-edge records.
// legal[v]: bit k when variant k can run v on a warp (0: not a warp vertex).
__global__ void k_features(const uint2 *__restrict__ row, const uint32_t *__restrict__ adj,
                           const uint32_t *__restrict__ rdeg, const uint64_t *__restrict__ work,
                           const uint64_t *__restrict__ inptr, uint32_t n, uint32_t warp_cap,
                           float *__restrict__ x, uint8_t *__restrict__ legal) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint2 rv = row[v];
    const uint32_t d = rv.y;
    const uint64_t nin = inptr[v + 1] - inptr[v];
    const uint32_t span = d ? adj[(uint64_t)rv.x * 4 + d - 1] - adj[(uint64_t)rv.x * 4] : 0u;
    const bool warp_fits = span <= bitmap_max_span(kWarpTableSlots) || d <= warp_cap;
    uint32_t lg = 0;
    if (d && nin && warp_fits)
      for (uint32_t k = 0; k < 4; ++k)
        if (variant_legal(k, d, span)) lg |= 1u << k;
    legal[v] = (uint8_t)lg;
    const float x0 = log2f(1.f + (float)rdeg[v]);
    const float x1 = log2f(1.f + (float)work[v] / (float)(nin ? nin : 1));
    float *xv = x + v * kMlpIn;
    xv[0] = x0;
    xv[1] = x1;
    xv[2] = x0 - x1;
    xv[3] = log2f(1.f + (float)d);
    xv[4] = log2f(1.f + (float)span);
    xv[5] = log2f(1.f + (float)nin);
  }
}

// The cost model over every warp vertex: variant = argmin over legal
// variants of predicted log2 cycles, pcost = predicted cycles of that variant.
__global__ void k_predict(const float *__restrict__ params, const float *__restrict__ x,
                          const uint8_t *__restrict__ legal, uint32_t n, uint8_t *__restrict__ variant,
                          uint64_t *__restrict__ pcost) {
  __shared__ float P[kMlpParams];
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) P[i] = params[i];
  __syncthreads();
  float h1[kMlpH1], h2[kMlpH2];
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t lg = legal[v];
    if (!lg) {
      variant[v] = 0xFF;
      pcost[v] = 0;
      continue;
    }
    float xi[kMlpIn], y[kMlpOut];
#pragma unroll
    for (int f = 0; f < kMlpIn; ++f) xi[f] = (x[v * kMlpIn + f] - P[kMlpMuX + f]) / P[kMlpSdX + f];
    mlp_forward_one(P, xi, h1, h2, y);
    uint32_t best = 0xFF;
    float by = 0.f;
#pragma unroll
    for (int k = 0; k < kMlpOut; ++k) {
      const float yk = y[k] * P[kMlpSdY + k] + P[kMlpMuY + k];
      if (((lg >> k) & 1) && (best == 0xFF || yk < by)) {
        best = k;
        by = yk;
      }
    }
    variant[v] = (uint8_t)best;
    pcost[v] = (uint64_t)exp2f(fminf(fmaxf(by, 0.f), 40.f));
  }
}

namespace {

int build_in_index(gary_graph *g, cudaStream_t s, InIndex &in) {
  const uint32_t n = g->n;
  const uint64_t W = g->dag.words;
  if (W >= (1ull << 32)) {
    set_error("graph too large for the in-edge index (%llu padded words)", (unsigned long long)W);
    return GARY_ERR_UNSUPPORTED;
  }
  ScratchAlloc pol_alloc{s};
  auto pol = thrust::cuda::par_nosync(pol_alloc).on(s);
  DevBuf<uint32_t> keys, keys2;
  DevBuf<uint2> vals, vals2;
  {
    DevBuf<uint32_t> rowid;
    GARY_TRY(padded_rowid(g->dag, rowid, s));
    GARY_TRY(keys.alloc(W, s));
    GARY_TRY(vals.alloc(W, s));
    k_in_candidates<<<grid_for(W), kThreads, 0, s>>>(g->dag.row.p, g->dag.adj.p, rowid.p, W, n, keys.p,
                                                     vals.p);
    GARY_CUDA(cudaGetLastError());
  }
  GARY_TRY(keys2.alloc(W, s));
  GARY_TRY(vals2.alloc(W, s));
  {
    cub::DoubleBuffer<uint32_t> kb(keys.p, keys2.p);
    cub::DoubleBuffer<uint2> vb(vals.p, vals2.p);
    size_t tmp = 0;
    const int eb = bits_for((uint64_t)n);  // keys <= n - 1
    GARY_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, kb, vb, W, 0, eb, s));
    DevBuf<uint8_t> t;
    GARY_TRY(t.alloc(tmp, s));
    GARY_CUDA(cub::DeviceRadixSort::SortPairs(t.p, tmp, kb, vb, W, 0, eb, s));
    if (kb.Current() != keys.p) std::swap(keys, keys2);
    if (vb.Current() != vals.p) std::swap(vals, vals2);
  }
  keys2.release();
  vals2.release();
  // records = number of keys < n - 1 (the rest carry the "no record" key n - 1)
  uint64_t m = 0;
  {
    DevBuf<uint64_t> pos;
    GARY_TRY(pos.alloc(1, s));
    k_first_geq<<<1, 1, 0, s>>>(keys.p, W, n - 1, pos.p);
    GARY_CUDA(cudaGetLastError());
    GARY_CUDA(cudaMemcpyAsync(&m, pos.p, 8, cudaMemcpyDeviceToHost, s));
    GARY_CUDA(cudaStreamSynchronize(s));
  }
  in.records = m;
  GARY_TRY(in.inptr.alloc_persistent((uint64_t)n + 1));
  thrust::fill(pol, in.inptr.p, in.inptr.p + n + 1, m);
  if (m) k_in_heads<<<grid_for(m), kThreads, 0, s>>>(keys.p, m, in.inptr.p);
  auto rb = thrust::make_reverse_iterator(in.inptr.p + n + 1);
  thrust::inclusive_scan(pol, rb, rb + n + 1, rb, MinU64());
  GARY_TRY(in.inedge.alloc_persistent(std::max<uint64_t>(m, 1)));
  if (m)
    GARY_CUDA(cudaMemcpyAsync(in.inedge.p, vals.p, m * sizeof(uint2), cudaMemcpyDeviceToDevice, s));
  GARY_TRY(in.work.alloc_persistent(n));
  GARY_CUDA(cudaMemsetAsync(in.work.p, 0, (uint64_t)n * 8, s));
  if (m)
    k_in_work<<<grid_for(m), kThreads, 0, s>>>(keys.p, vals.p, m,
                                              reinterpret_cast<unsigned long long *>(in.work.p));
  GARY_CUDA(cudaGetLastError());
  in.total_work = thrust::reduce(pol, in.work.p, in.work.p + n, 0ull);
  return GARY_OK;
}

}  // namespace

PlanParams resolve_params(PlanParams pp, uint64_t total_work) {
  // Measured on RMAT 18-24: the best warp tile holds about 1/32 of a resident
  // warp's share of the work (2^11 probes at RMAT-18 up to 2^15 at RMAT-22 and
  // above; larger tiles leave warps idle at the end, smaller ones pay the
  // per-tile cost), and three resident CTAs per SM (12 warps each, against two
  // of 16) pay from about 2^31 probes (RMAT-22) on.
  if (pp.min_blocks != 2 && pp.min_blocks != 3) pp.min_blocks = total_work >= (1ull << 31) ? 3 : 2;
  if (!pp.warp_tile_cost) {
    const uint64_t slots = (uint64_t)sm_count() * tc_warps(pp.min_blocks) * pp.min_blocks;
    const uint64_t want = total_work / (slots * 32);
    uint64_t t = 1ull << 11;
    while (t < want && t < (1ull << 15)) t <<= 1;
    pp.warp_tile_cost = t;
  }
  return pp;
}

int build_k3_plan(gary_graph *g, const PlanParams &pp_in, cudaStream_t s, gary_count_plan **out,
                  const float *model) {
  auto plan = std::make_unique<gary_count_plan>();
  const uint32_t n = g->n;
  ScratchAlloc pol_alloc{s};
  auto pol = thrust::cuda::par_nosync(pol_alloc).on(s);
  PhaseTrace tr("triangle plan", s);
  GARY_TRY(build_in_index(g, s, plan->in));
  tr.mark("in-edge index");
  const PlanParams pp = resolve_params(pp_in, plan->in.total_work);
  plan->params = pp;
  GARY_TRY(plan->vclass.alloc_persistent(n));
  DevBuf<uint64_t> costV;  // cost of each light vertex, 0 for the others
  DevBuf<uint32_t> kW, kC;
  GARY_TRY(costV.alloc(n, s));
  GARY_TRY(kW.alloc((uint64_t)n + 1, s));
  GARY_TRY(kC.alloc((uint64_t)n + 1, s));
  // learned plans: per-vertex features -> cost model -> variant and predicted cycles
  DevBuf<uint64_t> pcost;
  uint64_t tw = pp.warp_tile_cost;
  if (model) {
    DevBuf<float> x, dmodel;
    DevBuf<uint8_t> legal;
    GARY_TRY(x.alloc((uint64_t)n * kMlpIn, s));
    GARY_TRY(legal.alloc(n, s));
    GARY_TRY(dmodel.alloc(kMlpParams, s));
    GARY_TRY(pcost.alloc(n, s));
    GARY_TRY(plan->variant.alloc_persistent(n));
    GARY_CUDA(cudaMemcpyAsync(dmodel.p, model, kMlpParams * 4, cudaMemcpyHostToDevice, s));
    k_features<<<grid_for(n), kThreads, 0, s>>>(g->dag.row.p, g->dag.adj.p, g->rdeg.p, plan->in.work.p,
                                                plan->in.inptr.p, n, pp.warp_cap, x.p, legal.p);
    k_predict<<<grid_for(n), 128, 0, s>>>(dmodel.p, x.p, legal.p, n, plan->variant.p, pcost.p);
    GARY_CUDA(cudaGetLastError());
    const uint64_t total = thrust::reduce(pol, pcost.p, pcost.p + n, 0ull);
    // about 32 warp tiles per resident warp, in predicted cycles
    const uint64_t slots = (uint64_t)sm_count() * pp.min_blocks * tc_warps(pp.min_blocks) * 32;
    tw = std::max<uint64_t>(total / std::max<uint64_t>(slots, 1), 4096);
    plan->learned = true;
  }
  k_classify<<<grid_for(n), kThreads, 0, s>>>(g->dag.row.p, g->dag.adj.p, plan->in.work.p, plan->in.inptr.p, n, pp,
                                              model ? pcost.p : nullptr, tw, plan->vclass.p, costV.p, kW.p,
                                              kC.p);
  GARY_CUDA(cudaGetLastError());
  GARY_CUDA(cudaMemsetAsync(kW.p + n, 0, 4, s));
  GARY_CUDA(cudaMemsetAsync(kC.p + n, 0, 4, s));
  const uint64_t totalL = thrust::reduce(pol, costV.p, costV.p + n, 0ull);
  thrust::exclusive_scan(pol, kW.p, kW.p + n + 1, kW.p, 0u);
  thrust::exclusive_scan(pol, kC.p, kC.p + n + 1, kC.p, 0u);
  uint32_t nW = 0, nC = 0;
  GARY_CUDA(cudaMemcpyAsync(&nW, kW.p + n, 4, cudaMemcpyDeviceToHost, s));
  GARY_CUDA(cudaMemcpyAsync(&nC, kC.p + n, 4, cudaMemcpyDeviceToHost, s));
  GARY_CUDA(cudaStreamSynchronize(s));
  tr.mark("classify");
  const uint64_t G = totalL ? (totalL + tw - 1) / tw : 0;
  const uint64_t total = (uint64_t)nC + nW + G;
  if (total >= (1ull << 31)) {
    set_error("tile plan too large (%llu tiles)", (unsigned long long)total);
    return GARY_ERR_UNSUPPORTED;
  }
  plan->n_cta = nC;
  plan->n_warp = (uint32_t)(nW + G);
  GARY_TRY(plan->tiles.alloc_persistent(std::max<uint64_t>(total, 1)));
  k_fill_split_tiles<<<grid_for(n), kThreads, 0, s>>>(plan->in.inptr.p, n, kC.p, plan->tiles.p);
  k_fill_split_tiles<<<grid_for(n), kThreads, 0, s>>>(plan->in.inptr.p, n, kW.p,
                                                     plan->tiles.p + nC);
  GARY_CUDA(cudaGetLastError());
  if (G) {
    // light vertices in id order, and the exclusive prefix of their costs
    GARY_TRY(plan->light.alloc_persistent(n));
    const uint32_t L = (uint32_t)(thrust::copy_if(pol, thrust::counting_iterator<uint32_t>(0),
                                                  thrust::counting_iterator<uint32_t>(n),
                                                  plan->light.p, IsLight{plan->vclass.p}) -
                                  plan->light.p);
    plan->n_light = L;
    DevBuf<uint64_t> lc;
    GARY_TRY(lc.alloc((uint64_t)L + 1, s));
    auto costs = thrust::make_transform_iterator(plan->light.p, LightCost{costV.p});
    thrust::exclusive_scan(pol, costs, costs + L, lc.p, 0ull);
    DevBuf<uint32_t> starts;
    GARY_TRY(starts.alloc(G, s));
    auto targets = thrust::make_transform_iterator(thrust::counting_iterator<uint64_t>(0),
                                                   GroupTarget{tw});
    thrust::lower_bound(pol, lc.p, lc.p + L, targets, targets + G, starts.p);
    k_fill_group_tiles<<<grid_for(G), kThreads, 0, s>>>(starts.p, G, L, plan->tiles.p + nC + nW);
    GARY_CUDA(cudaGetLastError());
  }
  GARY_TRY(plan->sched.alloc_persistent(1));
  GARY_CUDA(cudaStreamSynchronize(s));
  tr.mark("tiles");
  *out = plan.release();
  return GARY_OK;
}

// ---------------------------------------------------------------------------
// Counting kernel
namespace {

constexpr uint32_t kWarpBitmapSpan = bitmap_max_span(kWarpTableSlots);  // ids a warp bitmap covers

// One chunk of at most 32 in-edge records [kb, ke): count the members of each
// suffix that `set` holds.  Suffixes are read as 32-byte-aligned octets of
// ids (two 16-byte loads from one sector); the lanes walk the concatenation of
// the chunk's octets, so short suffixes do not idle lanes.  Lists start on
// 32-byte boundaries and are padded with kSentinel to a multiple of 8 words,
// so an octet only ever holds words of its own list: ids up to and including
// v before the suffix (all below min N+(v)) and padding.  Every set rejects
// both as out of its [lo, lo + span] range, so no per-id mask is needed.
// All 32 lanes must call.
template <typename Set>
__device__ __forceinline__ uint32_t probe_octet(const uint4 &a, const uint4 &b, const Set &set) {
  return set.contains(a.x) + set.contains(a.y) + set.contains(a.z) + set.contains(a.w) +
         set.contains(b.x) + set.contains(b.y) + set.contains(b.z) + set.contains(b.w);
}

template <typename Set>
__device__ __forceinline__ uint32_t walk_chunk(const uint4 *__restrict__ adj4,
                                               const uint2 *__restrict__ edges, uint64_t kb,
                                               uint64_t ke, int lane, const Set &set) {
  const uint64_t kk = kb + lane;
  uint32_t o0 = 0, no = 0;
  if (kk < ke) {
    const uint2 r = edges[kk];
    o0 = r.x >> 3;
    no = ((r.x + r.y + 7) >> 3) - o0;
  }
  const uint32_t incl = warp_inclusive_sum(no, lane);
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  if (total == 0) return 0;
  // flattened position p of record k's octets maps to octet (o0 - excl) + p
  const uint32_t excl = incl - no;
  const uint32_t bias = o0 - excl;
  // Every record has octets (a suffix is never empty); only the lanes past
  // the last record have none, so the owners follow from the record starts.
  WarpOwners owners(excl, lane);
  auto fetch = [&](uint32_t pb, uint4 &a, uint4 &b) {
    const uint32_t own = owners.owner(pb);
    const uint32_t p = pb + lane;
    const uint32_t oc = __shfl_sync(kFull, bias, own) + p;
    if (p < total) {
      a = adj4[2 * oc];
      b = adj4[2 * oc + 1];
    } else {
      a = b = make_uint4(kSentinel, kSentinel, kSentinel, kSentinel);
    }
  };
  uint32_t cnt = 0;
  // two batches in flight: the next octet loads while this one is probed
  uint4 ca, cb;
  fetch(0, ca, cb);
  for (uint32_t pb = 32; pb < total; pb += 32) {
    uint4 na, nb;
    fetch(pb, na, nb);
    cnt += probe_octet(ca, cb, set);
    ca = na;
    cb = nb;
  }
  cnt += probe_octet(ca, cb, set);
  return cnt;
}

template <typename Set>
__device__ __forceinline__ uint32_t walk_range(const uint4 *__restrict__ adj4,
                                               const uint2 *__restrict__ edges, uint64_t kb,
                                               uint64_t ke, int lane, const Set &set) {
  uint32_t cnt = 0;
  for (uint64_t k = kb; k < ke; k += 32) cnt += walk_chunk(adj4, edges, k, ke, lane, set);
  return cnt;
}

// CTA tile: N+(v) does not fit a warp's set.  All warps share one set in the
// whole shared buffer and claim 32-record chunks of the tile dynamically.
template <int WARPS, typename Set>
__device__ __forceinline__ uint32_t cta_walk(const uint4 *__restrict__ adj4,
                                             const uint2 *__restrict__ edges, uint64_t kb,
                                             uint64_t ke, uint32_t *chunk, int lane,
                                             const Set &set) {
  uint32_t cnt = 0;
  while (true) {
    uint32_t c = 0;
    if (lane == 0) c = atomicAdd(chunk, 1u);
    c = __shfl_sync(kFull, c, 0);
    const uint64_t k = kb + (uint64_t)c * 32;
    if (k >= ke) break;
    cnt += walk_chunk(adj4, edges, k, ke < k + 32 ? ke : k + 32, lane, set);
  }
  return cnt;
}

// How CTA tiles hold N+(v): `words` shared words for the set (a multiple of
// 4, at most the CTA's buffer) and the poll limit of the first wait for a
// staging copy.
struct CtaSetCfg {
  uint32_t words;
  uint32_t polls;
};

// One CTA tile.  N+(v) goes into the cheapest set that fits `cfg.words`
// shared words: a bitmap of its id span, 4-slot hash buckets (d <= words/2),
// the sorted list staged whole by a bulk copy (d <= words; searched in
// shared memory only), or `words` evenly spaced samples of the list for the
// two-phase search (phase 2 in HBM).  Adds the tile's count to cnt_total.
// Returns false when a staging copy did not land within the drain wait: the
// CTA must then stop touching shared memory (the copy may still arrive), so
// the caller abandons its remaining work; the error word records it.
template <int WARPS>
__device__ bool cta_tile(const GraphView &g, const uint2 *__restrict__ inedge,
                         const uint64_t *__restrict__ inptr, const Tile &t, uint32_t *smem,
                         uint32_t *chunk, uint64_t *bar, uint32_t &phase, const CtaSetCfg &cfg,
                         SchedState *sched, const uint32_t *gid, unsigned long long *gcount,
                         unsigned long long &cnt_total) {
  const uint32_t S = cfg.words;
  const int lane = threadIdx.x & 31;
  const uint32_t v = t.v0;
  const uint2 rv = g.row[v];
  const uint32_t d = rv.y;
  const uint32_t *av = g.adj + (uint64_t)rv.x * 4;
  const uint4 *adj4 = reinterpret_cast<const uint4 *>(g.adj);
  const uint64_t base = inptr[v];
  const uint64_t kb = base + t.j0, ke = base + t.j1;
  const uint32_t lo = av[0], span = av[d - 1] - lo;
  auto sync = [] { __syncthreads(); };
  if (threadIdx.x == 0) *chunk = 0;
  uint32_t cnt = 0, path;
  if (span <= bitmap_max_span(S)) {
    path = kPathBitmap;
    const BitmapSet st = build_bitmap(av, d, lo, span, smem, threadIdx.x, blockDim.x, sync);
    cnt = cta_walk<WARPS>(adj4, inedge, kb, ke, chunk, lane, st);
  } else if (2 * d <= S) {
    path = kPathBuckets;
    const BucketSet st =
        build_buckets(av, d, lo, span, smem, S, threadIdx.x, blockDim.x, sync, &sched->error);
    cnt = cta_walk<WARPS>(adj4, inedge, kb, ke, chunk, lane, st);
  } else {
    if (d <= S) {
      // the whole list by one bulk copy (lists start 32-byte aligned and are
      // padded to whole octets, so the 16-byte-rounded size stays in the list)
      path = kPathStaged;
      if (threadIdx.x == 0) bulk_stage(smem, av, ((d + 3) / 4) * 16, bar);
      bool ok = mbar_wait_bounded(bar, phase, cfg.polls);
      if (!ok) {
        atomicOr(&sched->error, kLaunchErrStageWait);
        ok = mbar_wait_bounded(bar, phase);  // drain the copy before going on
      }
      if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) atomicOr(&sched->error, kLaunchErrStageDrain);
        return false;
      }
      phase ^= 1;
    } else {
      path = kPathSampled;
      for (uint32_t i = threadIdx.x; i < S; i += blockDim.x) smem[i] = av[(uint64_t)i * d / S];
      __syncthreads();
    }
    const SearchSet st{av, smem, d, S, lo, span};
    cnt = cta_walk<WARPS>(adj4, inedge, kb, ke, chunk, lane, st);
  }
  if (threadIdx.x == 0) atomicAdd(&sched->cta_path[path], 1u);
  if (gcount) {
    const unsigned long long tw = warp_sum_u64(cnt);
    if (lane == 0 && tw) atomicAdd(&gcount[gid[v]], tw);
  }
  cnt_total += cnt;
  // the next tile rewrites shared memory, possibly through the async proxy
  fence_proxy_async_smem();
  __syncthreads();
  return true;
}

// Sorted copy of N+(v) in shared memory, binary-searched (variant SEARCH).
struct SmemSearchSet {
  const uint32_t *list;
  uint32_t d, lo, span;
  __device__ __forceinline__ uint32_t contains(uint32_t x) const {
    if (x - lo > span) return 0;
    uint32_t b = 0, e = d;
    while (b < e) {
      const uint32_t m = (b + e) >> 1;
      const uint32_t v = list[m];
      if (v == x) return 1;
      if (v < x) b = m + 1;
      else e = m;
    }
    return 0;
  }
};

// Up to 8 ids held in registers in every lane, each probe compared against
// all of them (variant REGS).
struct RegSet8 {
  uint32_t r[8];
  __device__ __forceinline__ uint32_t contains(uint32_t x) const {
    uint32_t f = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) f |= (x == r[k]) ? 1u : 0u;
    return f;
  }
};

// Per-vertex control of the warp path; null pointers give the plain
// dispatch (bitmap when the span fits, else buckets) and no cycle log.
struct VertexCtl {
  const uint8_t *variant;      // intersection variant per middle vertex
  unsigned long long *cycles;  // clock64 cycles spent per middle vertex
  const uint32_t *gid;         // batches: graph of each middle vertex
  unsigned long long *gcount;  // batches: per-graph counts
  unsigned *err;               // the launch's error word
  unsigned long long *span;    // per CTA: start time, finish time of its last warp (ns)
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Batches: add a warp's count for middle vertex v to its graph's total.
__device__ __forceinline__ void add_graph_count(const VertexCtl &ctl, uint32_t v, uint32_t c,
                                                int lane) {
  if (!ctl.gcount) return;
  const unsigned long long t = warp_sum_u64(c);
  if (lane == 0 && t) atomicAdd(&ctl.gcount[ctl.gid[v]], t);
}

// One middle vertex v on one warp: a set of N+(v) in the warp's slots, walk
// in-edges [j0, j1) of v.
__device__ __forceinline__ uint32_t warp_vertex(const GraphView &g, const uint2 *__restrict__ inedge,
                                                const uint64_t *__restrict__ inptr, uint32_t v,
                                                uint32_t j0, uint32_t j1, uint32_t *tab, int lane,
                                                const VertexCtl &ctl) {
  const uint2 rv = g.row[v];
  const uint32_t d = rv.y;
  const uint64_t base = inptr[v];
  const uint64_t nin = inptr[v + 1] - base;
  const uint64_t ke = base + min_u64(j1, nin);
  const uint64_t kb = base + j0;
  if (d == 0 || kb >= ke) return 0;
  const long long t0 = ctl.cycles ? clock64() : 0;
  const uint32_t *av = g.adj + (uint64_t)rv.x * 4;
  const uint4 *adj4 = reinterpret_cast<const uint4 *>(g.adj);
  const uint32_t lo = av[0], span = av[d - 1] - lo;
  auto sync = [] { __syncwarp(); };
  uint32_t var = span <= kWarpBitmapSpan ? kVarBitmap : kVarHash;
  if (ctl.variant) {
    const uint32_t f = ctl.variant[v];
    if (variant_legal(f, d, span)) var = f;
  }
  uint32_t c;
  if (var == kVarBitmap) {
    const BitmapSet st = build_bitmap(av, d, lo, span, tab, lane, 32, sync);
    c = walk_range(adj4, inedge, kb, ke, lane, st);
  } else if (var == kVarHash) {
    const BucketSet st = build_buckets(av, d, lo, span, tab, kWarpTableSlots, lane, 32, sync, ctl.err);
    c = walk_range(adj4, inedge, kb, ke, lane, st);
  } else if (var == kVarSearch) {
    for (uint32_t i = lane; i < d; i += 32) tab[i] = av[i];
    __syncwarp();
    const SmemSearchSet st{tab, d, lo, span};
    c = walk_range(adj4, inedge, kb, ke, lane, st);
  } else {
    RegSet8 st;
#pragma unroll
    for (int k = 0; k < 8; ++k) st.r[k] = av[(uint32_t)k < d ? k : d - 1];  // repeats, never padding
    c = walk_range(adj4, inedge, kb, ke, lane, st);
  }
  __syncwarp();
  if (ctl.cycles && lane == 0) atomicAdd(&ctl.cycles[v], (unsigned long long)(clock64() - t0));
  add_graph_count(ctl, v, c, lane);
  return c;
}

template <int WARPS, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB)
    k_tc_mid(GraphView g, const uint2 *__restrict__ inedge, const uint64_t *__restrict__ inptr,
             const uint32_t *__restrict__ light, const Tile *__restrict__ tiles, uint32_t n_cta,
             TileRange rng, SchedState *sched, unsigned long long *__restrict__ out, VertexCtl ctl,
             CtaSetCfg cfg) {
  extern __shared__ __align__(16) uint32_t smem[];
  __shared__ uint64_t bar;
  __shared__ uint32_t s_tile, s_chunk;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long cnt = 0;

  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_fence_init();
    if (ctl.span) ctl.span[2 * blockIdx.x] = global_ns();
  }
  __syncthreads();
  uint32_t phase = 0;

  // phase 1: CTA tiles (N+(v) does not fit a warp's set)
  bool alive = true;
  while (true) {
    if (threadIdx.x == 0) s_tile = rng.cta_lo + atomicAdd(&sched->next_cta, 1u);
    __syncthreads();
    const uint32_t t = s_tile;
    __syncthreads();
    if (t >= rng.cta_hi) break;
    const Tile tl = tiles[t];
    if (!cta_tile<WARPS>(g, inedge, inptr, tl, smem, &s_chunk, &bar, phase, cfg, sched, ctl.gid,
                         ctl.gcount, cnt)) {
      alive = false;  // a staging copy may still land in shared memory: no more work here
      break;
    }
  }

  // phase 2: warp tiles, each warp on its own slots
  uint32_t *tab = smem + warp * kWarpTableSlots;
  const Tile *wt = tiles + n_cta;
  while (alive) {
    uint32_t t = 0;
    if (lane == 0) t = rng.warp_lo + atomicAdd(&sched->next_warp, 1u);
    t = __shfl_sync(kFull, t, 0);
    if (t >= rng.warp_hi) break;
    const Tile tl = wt[t];
    if (tl.j1 != kGroupTile) {
      cnt += warp_vertex(g, inedge, inptr, tl.v0, tl.j0, tl.j1, tab, lane, ctl);
      continue;
    }
    // a group of light vertices: list positions [v0, v1), 32 ids per load
    for (uint32_t ib = tl.v0; ib < tl.v1; ib += 32) {
      const uint32_t nb = min(32u, tl.v1 - ib);
      const uint32_t myv = lane < nb ? light[ib + lane] : 0u;
      for (uint32_t k = 0; k < nb; ++k)
        cnt += warp_vertex(g, inedge, inptr, __shfl_sync(kFull, myv, k), 0, 0xFFFFFFFFu, tab, lane,
                           ctl);
    }
  }

  cnt = warp_sum_u64(cnt);
  if (lane == 0 && cnt) atomicAdd(out, cnt);
  if (lane == 0 && ctl.span) atomicMax(&ctl.span[2 * blockIdx.x + 1], global_ns());
  if (threadIdx.x == 0 && alive) mbar_inval(&bar);
}

}  // namespace

int k3_features(gary_graph *g, gary_count_plan *plan, float *d_x, uint8_t *d_legal, cudaStream_t s) {
  k_features<<<grid_for(g->n), kThreads, 0, s>>>(g->dag.row.p, g->dag.adj.p, g->rdeg.p,
                                                 plan->in.work.p, plan->in.inptr.p, g->n,
                                                 plan->params.warp_cap, d_x, d_legal);
  GARY_CUDA(cudaGetLastError());
  return GARY_OK;
}

template <int MINB>
int launch_k3_impl(gary_graph *g, gary_count_plan *plan, unsigned long long *d_out, cudaStream_t s,
                   uint32_t shard, uint32_t nshards, VertexCtl ctl) {
  constexpr int WARPS = tc_warps(MINB);
  auto kern = k_tc_mid<WARPS, MINB>;
  const size_t smem = (size_t)WARPS * kWarpTableSlots * 4;
  static bool attr_done[64] = {false};
  const int dev = device_ordinal();
  if (dev < 64 && !attr_done[dev]) {
    GARY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr_done[dev] = true;
  }
  int per_sm = 0;
  GARY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, WARPS * 32, smem));
  if (per_sm < 1) per_sm = 1;
  const unsigned grid = (unsigned)std::min<int>(sm_count() * per_sm, (int)kMaxCountCtas);
  if (!plan->span.p) GARY_TRY(plan->span.alloc_persistent(2 * kMaxCountCtas));
  ctl.span = plan->span.p;
  const TileRange rng = shard_range(plan->n_cta, plan->n_warp, shard, nshards);
  const uint32_t words = (uint32_t)(WARPS * kWarpTableSlots);
  const uint32_t cw = plan->params.cta_set_words;
  const CtaSetCfg cfg{cw && cw < words ? cw : words, plan->params.stage_polls};
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  GARY_CUDA(cudaStreamIsCapturing(s, &cap));
  const bool timed = cap == cudaStreamCaptureStatusNone;
  GARY_CUDA(cudaMemsetAsync(plan->sched.p, 0, sizeof(SchedState), s));
  GARY_CUDA(cudaMemsetAsync(plan->span.p, 0, 2ull * grid * 8, s));
  GARY_CUDA(cudaMemsetAsync(d_out, 0, sizeof(unsigned long long), s));
  if (timed) GARY_CUDA(cudaEventRecord(g->ev0, s));
  kern<<<grid, WARPS * 32, smem, s>>>(g->view(), plan->in.inedge.p, plan->in.inptr.p, plan->light.p,
                                      plan->tiles.p, plan->n_cta, rng, plan->sched.p, d_out, ctl, cfg);
  GARY_CUDA(cudaGetLastError());
  if (timed) GARY_CUDA(cudaEventRecord(g->ev1, s));
  g->last = gary_count_stats{};
  g->last.tiles = (rng.cta_hi - rng.cta_lo) + (rng.warp_hi - rng.warp_lo);
  g->last.cta_tiles = rng.cta_hi - rng.cta_lo;
  g->last.work = plan->in.total_work;
  g->last_timed = timed;
  g->last_sched = plan->sched.p;
  g->last_span = plan->span.p;
  g->last_span_ctas = grid;
  return GARY_OK;
}

int launch_k3_ctl(gary_graph *g, gary_count_plan *plan, unsigned long long *d_out, cudaStream_t s,
                  uint32_t shard, uint32_t nshards, const uint8_t *variant,
                  unsigned long long *cycles, unsigned long long *gcount) {
  const VertexCtl ctl{variant, cycles, gcount ? g->gid.p : nullptr, gcount, &plan->sched.p->error, nullptr};
  if (plan->params.min_blocks >= 3) return launch_k3_impl<3>(g, plan, d_out, s, shard, nshards, ctl);
  return launch_k3_impl<2>(g, plan, d_out, s, shard, nshards, ctl);
}

int launch_k3(gary_graph *g, gary_count_plan *plan, unsigned long long *d_out, cudaStream_t s,
              uint32_t shard, uint32_t nshards) {
  return launch_k3_ctl(g, plan, d_out, s, shard, nshards, plan->variant.p, nullptr, nullptr);
}

}  // namespace gary
