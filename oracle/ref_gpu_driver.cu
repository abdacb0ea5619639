// Test infrastructure only: launches the REFERENCE's own triangle kernels
// (include/kernels/GraphQueryHom.cuh:15-43 and src/GraphQueryHom.cu:15-38,
// compiled in place for sm_100a by oracle/Makefile) on a graph uploaded by the
// reference's DeviceGraphCtx (src/DeviceGraph.cu:18-47).  Launch shapes follow
// test/TriQueryTest.cu:74-153: grid 1536 x block 256, dynamic shared memory
// getIndexCacheSMem(block, 32) * sizeof(vidT).
//
// This is the GPU half of the oracle: the reference's kernel built for
// Blackwell.  It is the bar the product kernels are compared against, for
// results (bit-exact) and for speed.  Nothing in the product links this file.
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>
#include <cuda_runtime.h>
#include <thrust/device_vector.h>

#include "Graph.h"
#include "DeviceGraph.cuh"
#include "kernels/GraphQueryHom.cuh"

namespace {
struct RefGpuGraph {
  DeviceGraphCtx ctx;
  thrust::device_vector<size_t> count64;
  thrust::device_vector<unsigned> count32;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};
thread_local char g_err[512];
int fail(cudaError_t e) {
  std::strncpy(g_err, cudaGetErrorString(e), sizeof(g_err) - 1);
  return -1;
}
}  // namespace

extern "C" {

const char *ref_gpu_last_error(void) { return g_err; }

// Upload a host CSR (any orientation the caller chose) through the
// reference's DeviceGraphCtx.  Returns an opaque handle or nullptr.
void *ref_gpu_graph_create(int32_t n, int64_t nnz, const int64_t *ptr, const int32_t *idx) {
  try {
    auto p = std::make_shared<std::vector<eidT>>(ptr, ptr + (size_t)n + 1);
    auto i = std::make_shared<std::vector<vidT>>(idx, idx + nnz);
    auto *g = new RefGpuGraph();
    g->ctx.loadFromHost(std::make_shared<GraphCSR>(n, nnz, p, i));
    g->ctx.populateDevice();
    g->count64.resize(1);
    g->count32.resize(1);
    cudaEventCreate(&g->ev0);
    cudaEventCreate(&g->ev1);
    return g;
  } catch (const std::exception &e) {
    std::strncpy(g_err, e.what(), sizeof(g_err) - 1);
    return nullptr;
  }
}

void ref_gpu_graph_free(void *h) {
  auto *g = static_cast<RefGpuGraph *>(h);
  if (!g) return;
  cudaEventDestroy(g->ev0);
  cudaEventDestroy(g->ev1);
  g->ctx.clear();
  delete g;
}

// variant: 0 = triangleCountHom<true,32,interleaved>  (TriQueryTest.cu:114-133)
//          1 = triangleCountHom<true,32,chunked>      (TriQueryTest.cu:135-153)
//          2 = triangleCountHom<false>                (TriQueryTest.cu:95-112)
//          3 = triangleCountLegacy (unsigned total)   (TriQueryTest.cu:74-93)
// Writes the count and the kernel time (CUDA events, default stream).
int ref_gpu_tri_count(void *h, int32_t variant, uint64_t *count, float *ms) {
  auto *g = static_cast<RefGpuGraph *>(h);
  constexpr int cacheSize = 32;
  dim3 grid(1536), block(256);
  DeviceGraph dg{g->ctx.getDeviceCSR(), g->ctx.getDeviceCOO()};
  size_t smem = graph_query::getIndexCacheSMem(block, cacheSize) * sizeof(vidT);
  cudaMemset(thrust::raw_pointer_cast(g->count64.data()), 0, sizeof(size_t));
  cudaMemset(thrust::raw_pointer_cast(g->count32.data()), 0, sizeof(unsigned));
  cudaEventRecord(g->ev0);
  switch (variant) {
    case 0:
      graph_query::triangleCountHom<true, cacheSize><<<grid, block, smem>>>(
          dg, thrust::raw_pointer_cast(g->count64.data()));
      break;
    case 1:
      graph_query::triangleCountHom<true, cacheSize, chunkedPolicy><<<grid, block, smem>>>(
          dg, thrust::raw_pointer_cast(g->count64.data()));
      break;
    case 2:
      graph_query::triangleCountHom<false><<<grid, block, 0>>>(
          dg, thrust::raw_pointer_cast(g->count64.data()));
      break;
    case 3:
      graph_query::triangleCountLegacy<<<grid, block, 0>>>(
          dg, thrust::raw_pointer_cast(g->count32.data()));
      break;
    default:
      std::strncpy(g_err, "unknown variant", sizeof(g_err) - 1);
      return -2;
  }
  cudaEventRecord(g->ev1);
  cudaError_t e = cudaEventSynchronize(g->ev1);
  if (e != cudaSuccess) return fail(e);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(e);
  cudaEventElapsedTime(ms, g->ev0, g->ev1);
  if (variant == 3) {
    unsigned c = 0;
    cudaMemcpy(&c, thrust::raw_pointer_cast(g->count32.data()), sizeof(c),
               cudaMemcpyDeviceToHost);
    *count = c;
  } else {
    size_t c = 0;
    cudaMemcpy(&c, thrust::raw_pointer_cast(g->count64.data()), sizeof(c),
               cudaMemcpyDeviceToHost);
    *count = c;
  }
  return 0;
}

}  // extern "C"
