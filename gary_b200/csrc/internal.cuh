// Internal declarations shared by the translation units of libgary_b200.so.
#pragma once
#include <cstdarg>
#include <cstdint>
#include <cstddef>
#include <cstdio>
#include <new>
#include <cuda_runtime.h>

#include "gary_b200.h"

namespace gary {

constexpr uint32_t kSentinel = 0xFFFFFFFFu;  // list padding; never a vertex id
constexpr int kWarp = 32;
constexpr unsigned kFull = 0xFFFFFFFFu;

// Bits of a counting launch's error word (SchedState::error), zeroed before
// every launch and read back by gary_count and gary_count_status.
enum : uint32_t {
  kLaunchErrStageWait = 1u,   // a bulk-copy wait gave up after its poll limit
  kLaunchErrStageDrain = 2u,  // the drain wait after it gave up too: that CTA stopped work
  kLaunchErrTableFull = 4u,   // a shared-memory table had no free slot (capacity rule broken)
};

// ---- error reporting (thread-local message; see gary_last_error) --------
void set_error(const char *fmt, ...);
void clear_error();

#define GARY_CUDA(expr)                                                              \
  do {                                                                               \
    cudaError_t _e = (expr);                                                         \
    if (_e != cudaSuccess) {                                                         \
      ::gary::set_error("%s (%s:%d): %s", #expr, __FILE__, __LINE__,                 \
                        cudaGetErrorString(_e));                                     \
      return _e == cudaErrorMemoryAllocation ? GARY_ERR_OOM : GARY_ERR_CUDA;         \
    }                                                                                \
  } while (0)

#define GARY_TRY(expr)               \
  do {                               \
    int _s = (expr);                 \
    if (_s != GARY_OK) return _s;    \
  } while (0)

#define GARY_CHECK_ARG(cond, ...)                \
  do {                                           \
    if (!(cond)) {                               \
      ::gary::set_error(__VA_ARGS__);            \
      return GARY_ERR_INVALID;                   \
    }                                            \
  } while (0)

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// ---- stream-ordered scratch pool -----------------------------------------
// One cudaMemPool per device, owned by the library, for the temporaries of
// graph construction and plan building.  Its release threshold (tuning key
// "pool_keep_bytes") is how much freed scratch the pool keeps mapped across
// synchronisations.  The default keeps all of it (a caching allocator: the
// next upload reuses the mapped pages); 0 hands everything back to the
// driver at each sync, and the next upload then pays to map its pages again
// (about 7x the upload time at 10^9 edges).
cudaMemPool_t scratch_pool();
void set_pool_keep_bytes(uint64_t bytes);

// Thrust temporaries from the scratch pool, stream-ordered on s.  Thrust's
// default allocator calls cudaMalloc / cudaFree, and cudaFree synchronises the
// whole device (a copy in flight on another stream included).  Use as
//   ScratchAlloc pol_alloc{s};
//   auto pol = thrust::cuda::par_nosync(pol_alloc).on(s);
// A failed allocation throws std::bad_alloc, which the C-ABI entry points
// turn into GARY_ERR_OOM.
struct ScratchAlloc {
  using value_type = char;
  cudaStream_t s;
  char *allocate(std::ptrdiff_t n) {
    void *p = nullptr;
    if (cudaMallocFromPoolAsync(&p, (size_t)n, scratch_pool(), s) != cudaSuccess) {
      cudaGetLastError();
      throw std::bad_alloc();
    }
    return static_cast<char *>(p);
  }
  void deallocate(char *p, size_t) { cudaFreeAsync(p, s); }
};

// ---- cached blocks for arrays that outlive a call -------------------------
// persistent_alloc hands out a cudaMalloc'd block (sizes rounded up: powers of
// two to 1 MiB, then 2 MiB steps), reusing a cached block of the same rounded
// size (up to 1/8 larger) when one is free.  persistent_free synchronises the
// block's device, as cudaFree does, so that no kernel still in flight can use
// the block, and then keeps it for the next allocation instead of returning
// it to the driver: an upload that follows a free of a graph of the same
// shape makes no driver allocation call at all.  Because a free synchronises
// the device, temporaries inside a call come from the scratch pool instead.  The cache shares the
// "pool_keep_bytes" limit with the scratch pool.  An allocation that finds
// the device full empties the cache and the scratch pool's free pages and
// tries once more.
cudaError_t persistent_alloc(void **p, size_t bytes);
void persistent_free(void *p);
void release_cached_memory();

// ---- phase trace (GARY_TRACE=1 in the environment) -----------------------
// mark() synchronises the stream and prints the wall time since the previous
// mark to stderr; with tracing off it does nothing and costs nothing.
struct PhaseTrace {
  const char *what;
  cudaStream_t s;
  bool on;
  double t0, t;
  PhaseTrace(const char *what, cudaStream_t s);
  void mark(const char *phase);
  ~PhaseTrace();
};

// ---- device buffer with RAII --------------------------------------------
// alloc(): stream-ordered temporary from the scratch pool (freed on the same
// stream).  alloc_persistent(): a cached block (persistent_alloc /
// persistent_free), for arrays that outlive the call and so must not depend
// on the caller's stream.
template <typename T>
struct DevBuf {
  T *p = nullptr;
  size_t n = 0;
  cudaStream_t s = nullptr;
  bool async = false;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  DevBuf(DevBuf &&o) noexcept : p(o.p), n(o.n), s(o.s), async(o.async) { o.p = nullptr; o.n = 0; }
  DevBuf &operator=(DevBuf &&o) noexcept {
    if (this != &o) {
      release();
      p = o.p; n = o.n; s = o.s; async = o.async;
      o.p = nullptr; o.n = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  int alloc(size_t count, cudaStream_t stream) { return alloc_(count, stream, true); }
  int alloc_persistent(size_t count) { return alloc_(count, nullptr, false); }
  void release() {
    if (p) {
      if (async) cudaFreeAsync(p, s);
      else persistent_free(p);
    }
    p = nullptr;
    n = 0;
  }
  size_t bytes() const { return n * sizeof(T); }

 private:
  int alloc_(size_t count, cudaStream_t stream, bool is_async) {
    release();
    s = stream;
    async = is_async;
    n = count;
    if (count == 0) return GARY_OK;
    cudaError_t e = is_async
        ? cudaMallocFromPoolAsync(reinterpret_cast<void **>(&p), count * sizeof(T),
                                  scratch_pool(), stream)
        : persistent_alloc(reinterpret_cast<void **>(&p), count * sizeof(T));
    if (e == cudaErrorMemoryAllocation && is_async) {  // cached blocks may hold the room
      cudaGetLastError();
      release_cached_memory();
      e = cudaMallocFromPoolAsync(reinterpret_cast<void **>(&p), count * sizeof(T), scratch_pool(), stream);
    }
    if (e != cudaSuccess) {
      p = nullptr;
      n = 0;
      cudaGetLastError();
      set_error("device allocation of %zu bytes failed: %s", count * sizeof(T),
                cudaGetErrorString(e));
      return e == cudaErrorMemoryAllocation ? GARY_ERR_OOM : GARY_ERR_CUDA;
    }
    return GARY_OK;
  }
};

// ---- kernel-side graph view: one 8-byte row record per vertex -----------
// row[v] = {off4, len}: v's list starts at adj + 4*off4 (32-byte aligned) and
// holds len ids, padded with kSentinel up to a multiple of 8.
// ranked: ids are degree ranks, so every list is in orientation order and
// N+(v) holds only ids > v.  Kernels use it to skip list prefixes that cannot
// close a pattern; with caller ids (GARY_KEEP_IDS) they must not.
struct GraphView {
  uint32_t n;
  const uint2 *__restrict__ row;
  const uint32_t *__restrict__ adj;
  bool ranked;
};

// grid sizing helper: a multiple of the SM count
int sm_count();
int device_ordinal();

}  // namespace gary
