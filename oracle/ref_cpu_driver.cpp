// Test infrastructure only: a C-ABI wrapper around the REFERENCE's own host
// graph code (include/Graph.h, src/Graph.cpp, compiled in place from the
// reference tree by oracle/Makefile) plus the reference's CPU triangle oracle.
//
// Used by tests/golden/make_golden.py to produce golden counts, by the
// `-m gpu` parity tests, and by bench.py's reference arm (the reference's CPU
// path timed on the host cores).  Nothing in the product links this file.
//
// Pipeline restated from convert.cpp:19-78 (convertCOO2CSR with symmetrize,
// then convertOrientCSR): COO -> symmetrize() -> toCSR_() -> toCOO() ->
// orientation() -> toCSR_().  All graph arithmetic is the reference's.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <vector>
#include <omp.h>

#include "Graph.h"
#include "ParUtils.h"

namespace {

thread_local char g_err[512];

void set_err(const char *what) {
  std::strncpy(g_err, what, sizeof(g_err) - 1);
  g_err[sizeof(g_err) - 1] = '\0';
}

// cpuTriCount restated from test/TriQueryTest.cu:17-37.  The only change is
// the accumulator width: the reference accumulates in `unsigned` (lines 17
// and 27) and truncates above 2^32; here both are uint64.  The set
// arithmetic (std::set_intersection into a scratch pad) is untouched.
// [v_begin, v_end) with stride lets bench.py time a bounded vertex sample.
uint64_t cpu_tri_count(const GraphCSR &csr, int64_t v_begin, int64_t v_end,
                       int64_t v_stride) {
  uint64_t count = 0;
  const auto &deg = csr.getDegreeAll();
  if (deg.empty()) return 0;
  vidT maxD = *std::max_element(deg.begin(), deg.end());
  std::vector<vidT> spad(std::max<vidT>(maxD, 1), 0);
  const int64_t nsteps = v_end > v_begin ? (v_end - v_begin + v_stride - 1) / v_stride : 0;

#pragma omp parallel for schedule(dynamic) firstprivate(spad)
  for (int64_t s = 0; s < nsteps; ++s) {
    const vidT v = (vidT)(v_begin + s * v_stride);
    const auto vAdj = csr.N(v);
    uint64_t localCount = 0;
    for (auto u : vAdj) {
      const auto uAdj = csr.N(u);
      auto outEnd = std::set_intersection(uAdj.begin(), uAdj.end(), vAdj.begin(),
                                          vAdj.end(), spad.begin());
      localCount += std::distance(spad.begin(), outEnd);
    }
    utils::atomicAdd(count, localCount);
  }
  return count;
}

}  // namespace

extern "C" {

const char *ref_last_error(void) { return g_err; }

// Oriented CSR built by the reference's own pipeline from an undirected edge
// list given once per edge (src[i], dst[i]); ids in [0, n).
void *ref_dag_from_edges(int32_t n, int64_t m, const int32_t *src, const int32_t *dst) {
  try {
    auto row = std::make_shared<std::vector<vidT>>(src, src + m);
    auto col = std::make_shared<std::vector<vidT>>(dst, dst + m);
    GraphCOO coo(n, m, row, col);
    GraphCOO sym = coo.symmetrize();
    GraphCSR csr = sym.toCSR_();
    GraphCOO dagCoo = csr.toCOO().orientation();
    return new GraphCSR(dagCoo.toCSR_());
  } catch (const std::exception &e) {
    set_err(e.what());
    return nullptr;
  }
}

// Symmetric CSR built by the reference pipeline (symmetrize -> toCSR_).
void *ref_sym_from_edges(int32_t n, int64_t m, const int32_t *src, const int32_t *dst) {
  try {
    auto row = std::make_shared<std::vector<vidT>>(src, src + m);
    auto col = std::make_shared<std::vector<vidT>>(dst, dst + m);
    GraphCOO coo(n, m, row, col);
    return new GraphCSR(coo.symmetrize().toCSR_());
  } catch (const std::exception &e) {
    set_err(e.what());
    return nullptr;
  }
}

// Wrap caller CSR arrays (copied) in the reference's GraphCSR.
void *ref_csr_from_arrays(int32_t n, int64_t nnz, const int64_t *ptr, const int32_t *idx) {
  try {
    auto p = std::make_shared<std::vector<eidT>>(ptr, ptr + (size_t)n + 1);
    auto i = std::make_shared<std::vector<vidT>>(idx, idx + nnz);
    return new GraphCSR(n, nnz, p, i);
  } catch (const std::exception &e) {
    set_err(e.what());
    return nullptr;
  }
}

int32_t ref_csr_num_v(void *h) { return static_cast<GraphCSR *>(h)->numV(); }
int64_t ref_csr_num_e(void *h) { return static_cast<GraphCSR *>(h)->numE(); }

void ref_csr_copy(void *h, int64_t *ptr, int32_t *idx) {
  auto *g = static_cast<GraphCSR *>(h);
  const auto &p = g->getPtr();
  const auto &i = g->getIdx();
  std::memcpy(ptr, p.data(), p.size() * sizeof(int64_t));
  std::memcpy(idx, i.data(), i.size() * sizeof(int32_t));
}

void ref_csr_free(void *h) { delete static_cast<GraphCSR *>(h); }

// The reference CPU triangle count over vertices v_begin, v_begin+stride, ...
// < v_end, using `threads` OpenMP threads (0 = the OpenMP default).
uint64_t ref_cpu_tri_count(void *h, int64_t v_begin, int64_t v_end, int64_t v_stride,
                           int32_t threads) {
  if (threads > 0) omp_set_num_threads(threads);
  if (v_stride < 1) v_stride = 1;
  return cpu_tri_count(*static_cast<GraphCSR *>(h), v_begin, v_end, v_stride);
}

int32_t ref_omp_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
