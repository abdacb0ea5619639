// Triangle count that allocates nothing on the device.
//
// For callers that cannot call cudaMalloc: code that runs while all device
// memory belongs to a host framework's own pool, or under a memory budget
// that forbids the library from growing its footprint.  They already hold the
// oriented graph on the device and pass it in; every other byte this path
// touches lives in one file-scope array, g_noalloc_scratch, which each GPU
// that loads the library holds until the process exits.
//
// Count: T = sum over u, over v in N+(u) of |N+(u) & N+(v)|, which counts
// each triangle once for any acyclic orientation (the reference's own formula,
// include/kernels/GraphQueryHom.cuh:15-43).  One warp per vertex u keeps
// N+(u) as a shared-memory bitmap or bucket set and walks the lists N+(v)
// with all lanes busy.  Lists need not be padded: reads are scalar.
//
// Scratch layout (unsigned long long words):
//   [0]                 next 32-vertex chunk (the work queue)
//   [1]                 reserved, zero
//   [2 + u / 2048]      partial count of the vertices of segment u / 2048
// so n may be at most 2048 * (16384 - 2) = 33,550,336 vertices.
#include <mutex>

#include "internal.cuh"
#include "warp_ops.cuh"

namespace gary {
namespace {

constexpr uint32_t kNoAllocWords = 16384;   // 128 KiB of scratch per GPU
constexpr uint32_t kNoAllocHeader = 2;
constexpr uint32_t kNoAllocSegment = 2048;  // vertices per partial-count word
constexpr uint64_t kNoAllocMaxN = (uint64_t)kNoAllocSegment * (kNoAllocWords - kNoAllocHeader);
constexpr int kNaWarps = 8;
constexpr uint32_t kNaSlots = 1024;  // shared words per warp

static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocWords];

std::mutex g_addr_mu;
unsigned long long *g_addr[64] = {};

// Device address of g_noalloc_scratch for the current device, fetched once
// per device with that device current.  (In host code the symbol itself is a
// host-side stand-in, not a device address.)
int scratch_address(unsigned long long **out) {
  int dev = 0;
  GARY_CUDA(cudaGetDevice(&dev));
  GARY_CHECK_ARG(dev >= 0 && dev < 64, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_addr_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    GARY_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_addr[dev] = static_cast<unsigned long long *>(p);
  }
  *out = g_addr[dev];
  return GARY_OK;
}

// N+(u) sorted in global memory: binary search (lists too long for the slots).
struct GlobalSearchSet {
  const uint32_t *list;
  uint32_t len, lo, span;
  __device__ __forceinline__ uint32_t contains(uint32_t x) const {
    if (x - lo > span) return 0;
    uint32_t b = 0, e = len;
    while (b < e) {
      const uint32_t mid = (b + e) >> 1;
      const uint32_t v = list[mid];
      if (v == x) return 1;
      if (v < x) b = mid + 1;
      else e = mid;
    }
    return 0;
  }
};

// Count, over v = au[j] for j < d, the members of N+(v) that `set` holds.
template <typename Set>
__device__ __forceinline__ uint32_t walk_out_lists(const uint64_t *__restrict__ indptr,
                                                   const uint32_t *__restrict__ colidx,
                                                   const uint32_t *__restrict__ deg, uint32_t n,
                                                   const uint32_t *__restrict__ au, uint32_t d,
                                                   int lane, const Set &set) {
  uint32_t cnt = 0;
  for (uint32_t j = 0; j < d; j += 32) {
    uint32_t len = 0;
    uint64_t start = 0;
    if (j + lane < d) {
      const uint32_t v = au[j + lane];
      if (v < n) {
        len = deg[v];
        start = indptr[v];
      }
    }
    const uint32_t incl = warp_inclusive_sum(len, lane);
    const uint32_t excl = incl - len;
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    WarpRuns own(excl, len, lane);
    for (uint32_t pb = 0; pb < total; pb += 32) {
      const uint32_t p = pb + lane;
      const int o = (int)own.owner(pb);
      const uint32_t ox = __shfl_sync(kFull, excl, o);
      const uint64_t os = __shfl_sync(kFull, start, o);
      if (p < total) cnt += set.contains(colidx[os + (p - ox)]);
    }
  }
  return cnt;
}

__global__ void __launch_bounds__(kNaWarps * 32)
    k_tc_noalloc(const uint64_t *__restrict__ indptr, const uint32_t *__restrict__ colidx,
                 const uint32_t *__restrict__ deg, uint32_t n) {
  __shared__ __align__(16) uint32_t smem[kNaWarps * kNaSlots];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t *tab = smem + warp * kNaSlots;
  unsigned long long *const queue = g_noalloc_scratch;
  unsigned long long *const partial = g_noalloc_scratch + kNoAllocHeader;
  auto sync = [] { __syncwarp(); };
  while (true) {
    unsigned long long c = 0;
    if (lane == 0) c = atomicAdd(queue, 1ull);
    c = __shfl_sync(kFull, c, 0);
    const uint64_t ub = c * 32;
    if (ub >= n) break;
    const uint64_t myu = ub + lane;
    const uint32_t myd = myu < n ? deg[myu] : 0u;
    unsigned todo = __ballot_sync(kFull, myd >= 2);
    while (todo) {
      const int k = __ffs(todo) - 1;
      todo &= todo - 1;
      const uint32_t u = (uint32_t)(ub + k);
      const uint32_t d = __shfl_sync(kFull, myd, k);
      const uint32_t *au = colidx + indptr[u];
      const uint32_t lo = au[0], span = au[d - 1] - lo;
      uint32_t cnt;
      if (span <= bitmap_max_span(kNaSlots)) {
        const BitmapSet st = build_bitmap(au, d, lo, span, tab, lane, 32, sync);
        cnt = walk_out_lists(indptr, colidx, deg, n, au, d, lane, st);
      } else if (2 * d <= kNaSlots) {
        const BucketSet st = build_buckets(au, d, lo, span, tab, kNaSlots, lane, 32, sync, nullptr);
        cnt = walk_out_lists(indptr, colidx, deg, n, au, d, lane, st);
      } else {
        const GlobalSearchSet st{au, d, lo, span};
        cnt = walk_out_lists(indptr, colidx, deg, n, au, d, lane, st);
      }
      __syncwarp();
      const unsigned long long sum = warp_sum_u64(cnt);
      if (lane == 0 && sum) atomicAdd(&partial[u / kNoAllocSegment], sum);
    }
  }
}

// *out = sum of the nseg partial counts (one CTA, fixed order per thread).
__global__ void k_noalloc_sum(uint32_t nseg, unsigned long long *__restrict__ out) {
  __shared__ unsigned long long red[32];
  const unsigned long long *partial = g_noalloc_scratch + kNoAllocHeader;
  unsigned long long x = 0;
  for (uint32_t i = threadIdx.x; i < nseg; i += blockDim.x) x += partial[i];
  x = warp_sum_u64(x);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = x;
  __syncthreads();
  if (threadIdx.x < 32) {
    x = threadIdx.x < blockDim.x / 32 ? red[threadIdx.x] : 0ull;
    x = warp_sum_u64(x);
    if (threadIdx.x == 0) *out = x;
  }
}

}  // namespace
}  // namespace gary

extern "C" int gary_count_triangles_noalloc(const uint64_t *d_indptr, const uint32_t *d_colidx,
                                            const uint32_t *d_deg, uint32_t n, void *stream,
                                            uint64_t *d_out) {
  using namespace gary;
  clear_error();
  GARY_CHECK_ARG(d_out != nullptr, "d_out is NULL");
  GARY_CHECK_ARG((uint64_t)n <= kNoAllocMaxN,
                 "n = %u exceeds the no-allocation limit of %llu vertices (scratch of %u words)", n,
                 (unsigned long long)kNoAllocMaxN, kNoAllocWords);
  GARY_CHECK_ARG(n == 0 || (d_indptr && d_colidx && d_deg), "graph pointers are NULL");
  cudaStream_t s = as_stream(stream);
  unsigned long long *scratch = nullptr;
  GARY_TRY(scratch_address(&scratch));
  const uint32_t nseg = (n + kNoAllocSegment - 1) / kNoAllocSegment;
  // every call starts from a cleared queue and cleared partial counts
  GARY_CUDA(cudaMemsetAsync(scratch, 0, (kNoAllocHeader + (size_t)nseg) * 8, s));
  if (n) {
    int per_sm = 0;
    GARY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tc_noalloc, kNaWarps * 32, 0));
    if (per_sm < 1) per_sm = 1;
    k_tc_noalloc<<<(unsigned)(sm_count() * per_sm), kNaWarps * 32, 0, s>>>(d_indptr, d_colidx,
                                                                          d_deg, n);
    GARY_CUDA(cudaGetLastError());
  }
  k_noalloc_sum<<<1, 256, 0, s>>>(nseg, reinterpret_cast<unsigned long long *>(d_out));
  GARY_CUDA(cudaGetLastError());
  return GARY_OK;
}
