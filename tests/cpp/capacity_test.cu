// Host-only check of the pattern kernels' capacity rules (pattern_rules.cuh):
// at every 4-clique out-degree the API admits, and on adversarial 4-cycle
// degree patterns, each worker's position hash or counter map stays at most
// half full, its counters cannot overflow, and its bit rows fit the buffer
// the plan gives them.  Exit status 0 when every check holds.
#include <cstdio>

#include "pattern_rules.cuh"

using namespace gary;

static int fails = 0, checks = 0;
#define CHECK(cond, ...)                                  \
  do {                                                    \
    ++checks;                                             \
    if (!(cond)) {                                        \
      ++fails;                                            \
      std::printf("FAIL line %d: ", __LINE__);            \
      std::printf(__VA_ARGS__);                           \
      std::printf("\n");                                  \
    }                                                     \
  } while (0)

static void k4_rules() {
  K4Worker prev = kK4None;
  for (uint32_t d = 0; d <= kK4MaxOutDegree; ++d) {
    const K4Worker w = k4_worker(d);
    CHECK(w >= prev, "d=%u: worker %d after %d (classes must grow with d)", d, w, prev);
    prev = w;
    if (d < 3) {
      CHECK(w == kK4None, "d=%u has no 4-clique but worker %d", d, w);
      continue;
    }
    // the hash gets 2^wanted slots unless the worker's table caps it: no cap
    // may happen, so every lookup meets a free slot
    CHECK(k4_wanted_log(d) <= k4_table_log(w), "d=%u: wants 2^%d slots, worker %d has 2^%d", d,
          k4_wanted_log(d), w, k4_table_log(w));
    CHECK(2ull * d <= (1ull << k4_table_log(w)), "d=%u: table more than half full", d);
    const uint64_t words = (uint64_t)d * k4_row_words(d);
    if (w == kK4Pool)
      CHECK(words > kK4BigRowWords, "d=%u: rows sent to HBM although %llu words fit shared memory", d,
            (unsigned long long)words);
    else
      CHECK(words <= k4_shared_row_words(w), "d=%u: %llu row words, worker %d has %u", d,
            (unsigned long long)words, w, k4_shared_row_words(w));
  }
  CHECK(k4_worker(kK4WarpMaxD) == kK4Warp && k4_worker(kK4WarpMaxD + 1) == kK4Mid, "warp/mid boundary");
  CHECK(k4_worker(kK4MidMaxD) == kK4Mid && k4_worker(kK4MidMaxD + 1) == kK4Big, "mid/big boundary");
  CHECK(k4_worker(877) == kK4Big && k4_worker(878) == kK4Pool, "shared/HBM row boundary at d+ = 877");
  // the HBM buffer of a CTA is sized for the graph's largest d+; every pool
  // vertex's rows must fit it
  uint32_t first_pool = kK4MidMaxD;
  while (k4_worker(first_pool) != kK4Pool) ++first_pool;
  for (uint32_t dmax : {first_pool, 1500u, 3124u, kK4MaxOutDegree}) {
    const uint64_t pool = (uint64_t)dmax * k4_row_words(dmax);
    for (uint32_t d = first_pool; d <= dmax; ++d)
      CHECK((uint64_t)d * k4_row_words(d) <= pool, "d=%u rows exceed the buffer sized for %u", d, dmax);
  }
}

static void c4_rules() {
  CHECK(c4_class(0, 0, 0) == kC4None && c4_class(0, 1u << 20, 1u << 20) == kC4None, "no lower neighbour");
  // Adversarial lower neighbourhoods: pre lower neighbours, each of degree k
  // (bound pre * k, the plan's sum of d(v)), and the exact wedge count anywhere
  // up to the bound.  The distinct w never exceed the wedges, and a count
  // c(u, w) never exceeds pre or the wedges (each v adds at most one to it).
  const uint32_t pres[] = {1, 2, 3, 31, 32, 33, 255, 256, 511, 512, 513, 4095, 8191, 8192, 8193, 65535, 65536, 1u << 20};
  const uint64_t ks[] = {1, 2, 3, 16, 511, 512, 513, 8191, 8192, 8193, 1u << 16, 1u << 24};
  for (uint32_t pre : pres)
    for (uint64_t k : ks) {
      const uint64_t bound = (uint64_t)pre * k;
      for (uint64_t exact : {bound, bound / 2, bound / 3 + 1, (uint64_t)kC4MidWedges, (uint64_t)kC4MidWedges + 1}) {
        if (exact > bound) continue;
        const C4Class c = c4_class(pre, bound, exact);
        const uint64_t distinct = exact;  // at most one w per wedge
        if (c == kC4Light) {
          CHECK(2 * bound <= kC4WarpSlots, "pre=%u k=%llu: light map over half full", pre, (unsigned long long)k);
          CHECK(2 * distinct <= kC4WarpSlots, "light distinct w");
        } else if (c == kC4Mid) {
          CHECK(2 * distinct <= kC4MidSlots, "pre=%u exact=%llu: mid map over half full", pre,
                (unsigned long long)exact);
          CHECK(exact < 65536, "pre=%u exact=%llu: 16-bit mid counts overflow", pre, (unsigned long long)exact);
          CHECK(bound > kC4LightWedges, "mid vertex with a light bound");
        } else {
          CHECK(c == kC4Heavy, "class");
          CHECK(exact > kC4MidWedges, "pre=%u exact=%llu: heavy below the mid limit", pre, (unsigned long long)exact);
          // window counters: 16 bits hold any count while pre fits them
          const uint64_t max_count = pre < exact ? pre : exact;
          if (!c4_wide_counters(pre)) CHECK(max_count <= 0xFFFFu, "pre=%u: 16-bit window counter overflow", pre);
        }
      }
    }
  CHECK(!c4_wide_counters(65535) && c4_wide_counters(65536), "16/32-bit window counter boundary");
  CHECK(c4_class(5, kC4LightWedges, kC4LightWedges) == kC4Light &&
            c4_class(5, kC4LightWedges + 1, kC4LightWedges + 1) == kC4Mid,
        "light/mid boundary");
  CHECK(c4_class(5, 1u << 20, kC4MidWedges) == kC4Mid && c4_class(5, 1u << 20, kC4MidWedges + 1) == kC4Heavy,
        "mid/heavy boundary");
}

int main() {
  k4_rules();
  c4_rules();
  std::printf("capacity rules: %d checks, %d failed\n", checks, fails);
  return fails ? 1 : 0;
}
