// Host-side entry points into the shim's search functions (include/gary/ops/
// Search.cuh is host+device code), so the CPU test suite can check them
// against the reference's own search results (tests/golden) without a GPU.
#include <cstdint>

#include "gary/ops/Search.cuh"

extern "C" {

// found[i] = binary_search(Span(list, n), keys[i])
void shim_binary_search(const uint32_t *list, uint64_t n, const uint32_t *keys, uint64_t nkeys,
                        uint8_t *found) {
  Span<const uint32_t, void> s(list, n);
  for (uint64_t i = 0; i < nkeys; ++i) found[i] = binary_search(s, keys[i]);
}

// found[i] / pos[i] = binary_search(Span(list, n), keys[i], pos)
void shim_binary_search_pos(const uint32_t *list, uint64_t n, const uint32_t *keys,
                            uint64_t nkeys, uint8_t *found, int32_t *pos) {
  Span<const uint32_t, void> s(list, n);
  for (uint64_t i = 0; i < nkeys; ++i) {
    int p = 0;
    found[i] = binary_search(s, keys[i], p);
    pos[i] = p;
  }
}

// the 32-entry cache of list, and found[i] = binary_search_2phase(list, cache, keys[i])
void shim_search_2phase(const uint32_t *list, uint64_t n, const uint32_t *keys, uint64_t nkeys,
                        uint32_t *cache_out, uint8_t *found) {
  Span<const uint32_t, void> s(list, n);
  uint32_t words[32];
  Array<uint32_t, 32> cache(words);
  build_cache(s, cache);
  for (int i = 0; i < 32; ++i) cache_out[i] = words[i];
  for (uint64_t i = 0; i < nkeys; ++i) found[i] = binary_search_2phase(s, cache, keys[i]);
}

}  // extern "C"
