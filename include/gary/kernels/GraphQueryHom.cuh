// Triangle-count kernels with the reference's names and launch contract: the
// shim of include/kernels/GraphQueryHom.cuh:13-48 and src/GraphQueryHom.cu:11-38.
//
// Two ways in:
//   1. Source-compatible kernels.  Callers launch them themselves, as the
//      reference's tests do (test/TriQueryTest.cu:114-127):
//        size_t smem = graph_query::getIndexCacheSMem(block, 32) * sizeof(vidT);
//        graph_query::triangleCountHom<true, 32><<<1536, 256, smem, s>>>(
//            ctx.getDeviceGraph(), d_count);
//      They sum |N(u) & N(v)| over the COO edges, one warp per edge, with the
//      set operations of gary/ops/Intersection.cuh.  Differences from the
//      reference: one atomic per warp instead of per thread; 64-bit edge
//      positions; and the legacy kernel reduces per warp rather than per block
//      (its unsigned total still wraps modulo 2^32, as the reference's does).
//   2. The library's own counting path (degree-oriented middle-vertex kernel,
//      persistent tile scheduler, cost-model variants) through the C ABI:
//        uint64_t t = graph_query::countTriangles(ctx);
//      This is the fast path; the kernels above exist so code written against
//      the reference's templates compiles unchanged.
//
// rectCountHom is only declared in the reference (GraphQueryHom.cuh:48);
// 4-cycles and 4-cliques are served here by countFourCycles /
// countFourCliques through the C ABI.
#pragma once
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "gary/DeviceGraph.cuh"
#include "gary/ops/DeviceIterator.cuh"
#include "gary/ops/Intersection.cuh"

namespace graph_query {

namespace cg = cooperative_groups;

// words of dynamic shared memory for `cacheSize` cache entries per warp
inline size_t getIndexCacheSMem(dim3 blockDim, size_t cacheSize) {
  return (size_t)warpsPerBlock(blockDim) * cacheSize;
}

namespace detail {
__device__ __forceinline__ unsigned long long warp_total(unsigned long long x) {
  for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(FULL_MASK, x, o);
  return x;
}
}  // namespace detail

// T = sum over COO edges (u, v) of |N(u) & N(v)|.  blockDim.x a multiple of
// 32; with useCache, dynamic shared memory of getIndexCacheSMem(blockDim, N)
// vidT words.  *count is accumulated into (zero it before the launch).
template <bool useCache = true, size_t N = 32, WorkPartition Policy = interleavedPolicy>
__global__ void triangleCountHom(DeviceGraph g, size_t *count) {
  extern __shared__ __align__(16) unsigned char gary_tc_smem[];
  auto block = cg::this_thread_block();
  auto warp = cg::tiled_partition<WARP_SIZE>(block);
  Array<vidT, N> cache(reinterpret_cast<vidT *>(gary_tc_smem) + N * warp.meta_group_rank());
  unsigned long long mine = 0;
  for (eidT e : g.coo.E().template cooperate<Policy>(warp, cg::this_grid())) {
    const vidT u = g.coo.rowIdx[e], v = g.coo.colIdx[e];
    if constexpr (useCache) mine += intersect(g.csr.N(u), g.csr.N(v), cache);
    else mine += intersect(g.csr.N(u), g.csr.N(v));
  }
  mine = detail::warp_total(mine);
  if (warp.thread_rank() == 0 && mine)
    atomicAdd(reinterpret_cast<unsigned long long *>(count), mine);
}

// The reference's legacy count (src/GraphQueryHom.cu:15-38): interleaved
// edges, a 32-entry cache per warp in static shared memory, an unsigned total.
// (static: a header-defined kernel gets one copy per translation unit.)
static __global__ void __launch_bounds__(1024) triangleCountLegacy(DeviceGraph g, unsigned *count) {
  __shared__ vidT cache[MAX_WARPS_PER_BLOCK * WARP_SIZE];
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x / WARP_SIZE);
  const uint64_t wid = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / WARP_SIZE;
  unsigned long long mine = 0;
  for (uint64_t e = wid; e < g.coo.nnz; e += warps) {
    const vidT u = g.coo.rowIdx[e], v = g.coo.colIdx[e];
    mine += intersect_bs_cache(const_cast<vidT *>(g.csr.colIdx + g.csr.indPtr[u]), g.csr.deg[u],
                               const_cast<vidT *>(g.csr.colIdx + g.csr.indPtr[v]), g.csr.deg[v],
                               cache);
  }
  mine = detail::warp_total(mine);
  if ((threadIdx.x & (WARP_SIZE - 1)) == 0 && mine) atomicAdd(count, (unsigned)mine);
}

// ---- the library's counting path ---------------------------------------
inline uint64_t countPattern(DeviceGraphCtx &ctx, int pattern, int sched = GARY_SCHED_PLAIN,
                             cudaStream_t stream = nullptr) {
  uint64_t out = 0;
  gary::check(gary_count(ctx.handle(), pattern, sched, stream, &out), "gary_count");
  return out;
}
inline uint64_t countTriangles(DeviceGraphCtx &ctx, int sched = GARY_SCHED_PLAIN,
                               cudaStream_t stream = nullptr) {
  return countPattern(ctx, GARY_PATTERN_TRIANGLE, sched, stream);
}
inline uint64_t countFourCycles(DeviceGraphCtx &ctx, cudaStream_t stream = nullptr) {
  return countPattern(ctx, GARY_PATTERN_4CYCLE, GARY_SCHED_PLAIN, stream);
}
inline uint64_t countFourCliques(DeviceGraphCtx &ctx, cudaStream_t stream = nullptr) {
  return countPattern(ctx, GARY_PATTERN_4CLIQUE, GARY_SCHED_PLAIN, stream);
}

}  // namespace graph_query
