// Internal declarations shared by the translation units of libgary_b200.so.
#pragma once
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

#include "gary_b200.h"

namespace gary {

constexpr uint32_t kSentinel = 0xFFFFFFFFu;  // list padding; never a vertex id
constexpr int kWarp = 32;
constexpr unsigned kFull = 0xFFFFFFFFu;

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
// stream).  alloc_persistent(): cudaMalloc / cudaFree, for arrays that outlive
// the call and so must not depend on the caller's stream.
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
      else cudaFree(p);
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
        : cudaMalloc(reinterpret_cast<void **>(&p), count * sizeof(T));
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
