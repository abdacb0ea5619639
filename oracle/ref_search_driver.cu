// Test infrastructure only: C-ABI wrappers that run the REFERENCE's own
// HOST_DEVICE search templates (include/ops/Search.cuh, compiled in place from
// the reference tree by oracle/Makefile) on the host, the way
// test/SearchTest.cu:235-257 does.  They produce golden vectors for the
// search semantics; nothing in the product links this file.
#include <cstdint>
#include <vector>

#include "ops/DeviceIterator.cuh"
#include "ops/Search.cuh"

extern "C" {

// binary_search(Span, key) -- include/ops/Search.cuh:48-61
void ref_binary_search(const int32_t *list, int64_t n, const int32_t *keys, int64_t nk,
                       uint8_t *found) {
  Span<const int32_t, void> span{list, (size_t)n};
  for (int64_t i = 0; i < nk; ++i) found[i] = binary_search(span, keys[i]) ? 1 : 0;
}

// binary_search(Span, key, pos) -- include/ops/Search.cuh:67-81; pos is the
// found index, or the insertion position minus one when absent.
void ref_binary_search_pos(const int32_t *list, int64_t n, const int32_t *keys, int64_t nk,
                           uint8_t *found, int32_t *pos) {
  Span<const int32_t, void> span{list, (size_t)n};
  for (int64_t i = 0; i < nk; ++i) {
    int p = 0;
    found[i] = binary_search(span, keys[i], p) ? 1 : 0;
    pos[i] = p;
  }
}

// build_cache -- include/ops/Search.cuh:93-100, N = 32
void ref_build_cache32(const int32_t *list, int64_t n, int32_t *cache) {
  Span<const int32_t, void> span{list, (size_t)n};
  Array<int32_t, 32> view{cache};
  build_cache(span, view);
}

// binary_search_2phase(Span, Array<32>, key) -- include/ops/Search.cuh:120-138,
// with the cache built by build_cache as test/SearchTest.cu:357-361 does.
void ref_binary_search_2phase(const int32_t *list, int64_t n, const int32_t *keys,
                              int64_t nk, uint8_t *found) {
  std::vector<int32_t> cache(32);
  Span<const int32_t, void> span{list, (size_t)n};
  Array<int32_t, 32> view{cache.data()};
  build_cache(span, view);
  for (int64_t i = 0; i < nk; ++i)
    found[i] = binary_search_2phase<const int32_t>(span, view, keys[i]) ? 1 : 0;
}

}  // extern "C"
