// End-to-end check of the C++ shim layer (include/gary/): code written the way
// the reference's test/TriQueryTest.cu and test/SetOpTest.cu use the
// reference's headers, compiled against the shims and linked to
// libgary_b200.so.
//
//   shim_test [scale] [edge_factor] [seed]
//
// Builds a seeded RMAT graph through the C ABI, orients it by id on the host
// (row u keeps its neighbours v < u, the reference's GraphCOO::orientation,
// src/Graph.cpp:34-61), loads it with DeviceGraphCtx::loadFromHost, launches
// the source-compatible kernels the way the reference's tests do (1536 x 256,
// cache of 32 per warp), runs the library's own counts, and checks the set
// operations on random pairs against std::set_intersection.  Prints one JSON
// line; exit status 0 only when every count and every pair agree.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <memory>
#include <random>
#include <vector>

#include "gary/Graph.h"
#include "gary/kernels/GraphQueryHom.cuh"
#include "gary/ops/Intersection.cuh"
#include "gary/ops/Search.cuh"

#define CK(x)                                                                  \
  do {                                                                         \
    cudaError_t e_ = (x);                                                      \
    if (e_ != cudaSuccess) {                                                   \
      std::fprintf(stderr, "%s: %s\n", #x, cudaGetErrorString(e_));            \
      std::exit(2);                                                            \
    }                                                                          \
  } while (0)

// the parts of the reference's GraphCSR (include/Graph.h:157-252) that
// DeviceGraphCtx::loadFromHost reads, with the reference's int64/int32 types
struct HostCSR {
  int32_t m = 0;
  std::vector<int64_t> ptr;
  std::vector<int32_t> idx;
  int32_t numV() const { return m; }
  int64_t numE() const { return (int64_t)idx.size(); }
  const std::vector<int64_t> &getPtr() const { return ptr; }
  const std::vector<int32_t> &getIdx() const { return idx; }
};

// per pair p: A = a[aoff[p] .. aoff[p]+alen[p]), B likewise; one warp per pair
template <bool Cached>
__global__ void k_pairs(const uint32_t *a, const uint64_t *aoff, const uint32_t *alen,
                        const uint32_t *b, const uint64_t *boff, const uint32_t *blen,
                        const uint64_t *ooff, uint32_t npairs, uint32_t *out, uint32_t *counts,
                        uint32_t *share_sums) {
  extern __shared__ __align__(16) unsigned char smem[];
  const uint32_t warp = threadIdx.x / WARP_SIZE, warps = blockDim.x / WARP_SIZE;
  Array<uint32_t, 32> cache(reinterpret_cast<uint32_t *>(smem) + 32 * warp);
  for (uint32_t p = blockIdx.x * warps + warp; p < npairs; p += gridDim.x * warps) {
    Span<const uint32_t, void> sA(a + aoff[p], alen[p]), sB(b + boff[p], blen[p]);
    int mine;
    if (Cached) mine = intersectBinarySearch(sA, sB, cache, out + ooff[p]);
    else mine = intersectBinarySearch(sA, sB, out + ooff[p]);
    // the count-only forms must give the same shares
    const int again = Cached ? intersect(sA, sB, cache) : intersect(sA, sB);
    unsigned long long tot = graph_query::detail::warp_total((unsigned long long)mine);
    unsigned long long tot2 = graph_query::detail::warp_total((unsigned long long)again);
    if ((threadIdx.x & 31) == 0) {
      counts[p] = (uint32_t)tot;
      share_sums[p] = (uint32_t)tot2;
    }
  }
}

// intersect_num with an upper bound and one ancestor, per pair (warp per pair)
__global__ void k_pairs_num(const uint32_t *a, const uint64_t *aoff, const uint32_t *alen,
                            const uint32_t *b, const uint64_t *boff, const uint32_t *blen,
                            const uint32_t *bound, const uint32_t *anc, uint32_t npairs,
                            uint32_t *counts) {
  const uint32_t warp = threadIdx.x / WARP_SIZE, warps = blockDim.x / WARP_SIZE;
  for (uint32_t p = blockIdx.x * warps + warp; p < npairs; p += gridDim.x * warps) {
    uint32_t *A = const_cast<uint32_t *>(a + aoff[p]), *B = const_cast<uint32_t *>(b + boff[p]);
    const uint32_t mine = intersect_num(A, alen[p], B, blen[p], bound[p], anc[p]);
    const unsigned long long tot = graph_query::detail::warp_total((unsigned long long)mine);
    if ((threadIdx.x & 31) == 0) counts[p] = (uint32_t)tot;
  }
}

// the warp-level two-phase search (Search.cuh:140-170 form): lane l searches keys[l + 32 k]
__global__ void k_search(const uint32_t *list, uint32_t n, const uint32_t *keys, uint32_t nkeys,
                         uint8_t *found) {
  __shared__ uint32_t cache[32 * 8];
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x / 32;
  cache[w * 32 + lane] = list[(uint64_t)lane * n / 32];
  __syncwarp();
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nkeys; i += gridDim.x * blockDim.x)
    found[i] = binary_search_2phase(const_cast<uint32_t *>(list), cache, keys[i], n);
}

static uint64_t cpu_count(const HostCSR &g) {
  uint64_t t = 0;
  std::vector<int32_t> tmp;
  for (int32_t u = 0; u < g.m; ++u)
    for (int64_t k = g.ptr[u]; k < g.ptr[u + 1]; ++k) {
      const int32_t v = g.idx[k];
      tmp.clear();
      std::set_intersection(g.idx.begin() + g.ptr[u], g.idx.begin() + g.ptr[u + 1],
                            g.idx.begin() + g.ptr[v], g.idx.begin() + g.ptr[v + 1],
                            std::back_inserter(tmp));
      t += tmp.size();
    }
  return t;
}

int main(int argc, char **argv) {
  const int scale = argc > 1 ? std::atoi(argv[1]) : 14;
  const int ef = argc > 2 ? std::atoi(argv[2]) : 8;
  const uint64_t seed = argc > 3 ? std::strtoull(argv[3], nullptr, 10) : 1;
  const uint32_t n = 1u << scale;
  const uint64_t samples = (uint64_t)ef << scale;

  // ---- graph through the C ABI, oriented by id on the host
  std::vector<uint32_t> src(samples), dst(samples);
  gary::check(gary_gen_rmat(scale, seed, 0, samples, src.data(), dst.data()), "gary_gen_rmat");
  gary_csr *csr = nullptr;
  gary::check(gary_csr_from_edges(src.data(), dst.data(), samples, n, 0, nullptr, &csr),
              "gary_csr_from_edges");
  uint32_t cn = 0;
  uint64_t nnz = 0;
  gary::check(gary_csr_info(csr, &cn, &nnz), "gary_csr_info");
  std::vector<uint64_t> sp(cn + 1);
  std::vector<uint32_t> si(nnz);
  gary::check(gary_csr_download(csr, sp.data(), si.data()), "gary_csr_download");
  gary_csr_free(csr);
  auto dag = std::make_shared<HostCSR>();
  dag->m = (int32_t)n;
  dag->ptr.assign(1, 0);
  for (uint32_t u = 0; u < n; ++u) {
    for (uint64_t k = sp[u]; k < sp[u + 1]; ++k)
      if (si[k] < u) dag->idx.push_back((int32_t)si[k]);
    dag->ptr.push_back((int64_t)dag->idx.size());
  }
  const uint64_t want = cpu_count(*dag);

  // ---- the reference's file round trip (saveToBinary / loadFromBinary) and
  // launch pattern over the shim views
  const std::string bin = std::string(std::getenv("TMPDIR") ? std::getenv("TMPDIR") : "/tmp") +
                          "/gary_shim_csr_dag_" + std::to_string(seed) + ".bin";
  {
    std::vector<eidT> p64(dag->ptr.begin(), dag->ptr.end());
    std::vector<vidT> i32(dag->idx.begin(), dag->idx.end());
    saveToBinary(GraphCSR(std::move(p64), std::move(i32)), bin);
  }
  auto loaded = loadFromBinary<GraphCSR>(bin);
  std::remove(bin.c_str());
  bool file_ok = loaded.numV() == (vidT)n && loaded.numE() == (eidT)dag->idx.size();
  for (size_t k = 0; file_ok && k < dag->idx.size(); ++k) file_ok = loaded.getIdx()[k] == (vidT)dag->idx[k];
  DeviceGraphCtx ctx;
  ctx.loadFromHost(std::make_shared<GraphCSR>(std::move(loaded)));
  ctx.populateDevice();
  const DeviceGraph dg = ctx.getDeviceGraph();
  size_t *d_count;
  unsigned *d_legacy;
  CK(cudaMalloc(&d_count, sizeof(size_t)));
  CK(cudaMalloc(&d_legacy, sizeof(unsigned)));
  const dim3 grid(1536), block(256);
  const size_t smem = graph_query::getIndexCacheSMem(block, 32) * sizeof(vidT);
  size_t got[3];
  for (int variant = 0; variant < 3; ++variant) {
    CK(cudaMemset(d_count, 0, sizeof(size_t)));
    if (variant == 0) graph_query::triangleCountHom<true, 32><<<grid, block, smem>>>(dg, d_count);
    if (variant == 1) graph_query::triangleCountHom<false><<<grid, block>>>(dg, d_count);
    if (variant == 2)
      graph_query::triangleCountHom<true, 32, chunkedPolicy><<<grid, block, smem>>>(dg, d_count);
    CK(cudaGetLastError());
    CK(cudaMemcpy(&got[variant], d_count, sizeof(size_t), cudaMemcpyDeviceToHost));
  }
  CK(cudaMemset(d_legacy, 0, sizeof(unsigned)));
  graph_query::triangleCountLegacy<<<grid, block>>>(dg, d_legacy);
  CK(cudaGetLastError());
  unsigned legacy = 0;
  CK(cudaMemcpy(&legacy, d_legacy, sizeof(unsigned), cudaMemcpyDeviceToHost));
  const uint64_t fast = graph_query::countTriangles(ctx);
  const uint64_t c4 = graph_query::countFourCycles(ctx);
  const uint64_t k4 = graph_query::countFourCliques(ctx);

  // the views: every list sorted, padded and 16-byte aligned; rows partition the COO
  std::vector<uint64_t> hp;
  std::vector<uint32_t> hi;
  ctx.getHostCSR(hp, hi);
  bool views_ok = file_ok && hp.size() == (size_t)n + 1 && hi.size() == dag->idx.size() &&
                  dg.csr.numE() == dg.coo.numE() && dg.coo.numE() == hi.size() &&
                  ((uintptr_t)dg.csr.colIdx & 15) == 0;

  // ---- set operations on random pairs (Zipf-like lengths, planted overlap)
  std::mt19937_64 rng(seed * 7919 + 17);
  const uint32_t npairs = 3000;
  std::vector<uint32_t> A, B, alen(npairs), blen(npairs);
  std::vector<uint64_t> aoff(npairs), boff(npairs), ooff(npairs);
  std::vector<std::vector<uint32_t>> expect(npairs);
  uint64_t osum = 0;
  for (uint32_t p = 0; p < npairs; ++p) {
    auto len = [&]() -> uint32_t {
      const double u = std::uniform_real_distribution<double>(0, 1)(rng);
      return (uint32_t)std::min(4000.0, std::pow(4001.0, u) - 1.0);
    };
    std::vector<uint32_t> a(len()), b(len());
    const uint32_t range = 1u + (uint32_t)(rng() % 20000);
    for (auto &x : a) x = (uint32_t)(rng() % range);
    for (auto &x : b) x = (uint32_t)(rng() % range);
    std::sort(a.begin(), a.end());
    a.erase(std::unique(a.begin(), a.end()), a.end());
    std::sort(b.begin(), b.end());
    b.erase(std::unique(b.begin(), b.end()), b.end());
    std::set_intersection(a.begin(), a.end(), b.begin(), b.end(), std::back_inserter(expect[p]));
    aoff[p] = A.size();
    alen[p] = (uint32_t)a.size();
    A.insert(A.end(), a.begin(), a.end());
    boff[p] = B.size();
    blen[p] = (uint32_t)b.size();
    B.insert(B.end(), b.begin(), b.end());
    ooff[p] = osum;
    osum += std::min(a.size(), b.size());
  }
  A.push_back(0);
  B.push_back(0);
  uint32_t *dA, *dB, *dal, *dbl, *dout, *dcnt, *dsh;
  uint64_t *dao, *dbo, *doo;
  CK(cudaMalloc(&dA, A.size() * 4));
  CK(cudaMalloc(&dB, B.size() * 4));
  CK(cudaMalloc(&dal, npairs * 4));
  CK(cudaMalloc(&dbl, npairs * 4));
  CK(cudaMalloc(&dao, npairs * 8));
  CK(cudaMalloc(&dbo, npairs * 8));
  CK(cudaMalloc(&doo, npairs * 8));
  CK(cudaMalloc(&dout, (osum + 1) * 4));
  CK(cudaMalloc(&dcnt, npairs * 4));
  CK(cudaMalloc(&dsh, npairs * 4));
  CK(cudaMemcpy(dA, A.data(), A.size() * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dB, B.data(), B.size() * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dal, alen.data(), npairs * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dbl, blen.data(), npairs * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dao, aoff.data(), npairs * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dbo, boff.data(), npairs * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(doo, ooff.data(), npairs * 8, cudaMemcpyHostToDevice));
  uint64_t pair_bad = 0;
  for (int cached = 0; cached < 2; ++cached) {
    CK(cudaMemset(dout, 0xFF, (osum + 1) * 4));
    if (cached)
      k_pairs<true><<<148, 256, 8 * 32 * 4>>>(dA, dao, dal, dB, dbo, dbl, doo, npairs, dout, dcnt, dsh);
    else
      k_pairs<false><<<148, 256>>>(dA, dao, dal, dB, dbo, dbl, doo, npairs, dout, dcnt, dsh);
    CK(cudaGetLastError());
    std::vector<uint32_t> out(osum + 1), cnt(npairs), sh(npairs);
    CK(cudaMemcpy(out.data(), dout, (osum + 1) * 4, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(cnt.data(), dcnt, npairs * 4, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(sh.data(), dsh, npairs * 4, cudaMemcpyDeviceToHost));
    for (uint32_t p = 0; p < npairs; ++p) {
      const auto &e = expect[p];
      bool ok = cnt[p] == e.size() && sh[p] == e.size();
      for (size_t k = 0; ok && k < e.size(); ++k) ok = out[ooff[p] + k] == e[k];
      pair_bad += !ok;
    }
  }

  // ---- bounded, ancestor-filtered counts against the host
  {
    std::vector<uint32_t> bound(npairs), anc(npairs), want(npairs);
    for (uint32_t p = 0; p < npairs; ++p) {
      bound[p] = (uint32_t)(rng() % 20001);
      const auto &e = expect[p];
      anc[p] = e.empty() ? 0u : e[rng() % e.size()];
      uint32_t c = 0;
      for (uint32_t x : e) c += x < bound[p] && x != anc[p];
      want[p] = c;
    }
    uint32_t *dbd, *dan;
    CK(cudaMalloc(&dbd, npairs * 4));
    CK(cudaMalloc(&dan, npairs * 4));
    CK(cudaMemcpy(dbd, bound.data(), npairs * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dan, anc.data(), npairs * 4, cudaMemcpyHostToDevice));
    k_pairs_num<<<148, 256>>>(dA, dao, dal, dB, dbo, dbl, dbd, dan, npairs, dcnt);
    CK(cudaGetLastError());
    std::vector<uint32_t> got(npairs);
    CK(cudaMemcpy(got.data(), dcnt, npairs * 4, cudaMemcpyDeviceToHost));
    for (uint32_t p = 0; p < npairs; ++p) pair_bad += got[p] != want[p];
  }

  // ---- warp-level two-phase search against std::binary_search
  std::vector<uint32_t> list(B.begin() + boff[0], B.begin() + boff[0] + blen[0]);
  for (uint32_t p = 1; list.size() < 100; ++p) list.assign(B.begin() + boff[p], B.begin() + boff[p] + blen[p]);
  std::vector<uint32_t> keys(20000);
  for (auto &k : keys) k = (uint32_t)(rng() % 21000);
  uint32_t *dl, *dk;
  uint8_t *df;
  CK(cudaMalloc(&dl, list.size() * 4));
  CK(cudaMalloc(&dk, keys.size() * 4));
  CK(cudaMalloc(&df, keys.size()));
  CK(cudaMemcpy(dl, list.data(), list.size() * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dk, keys.data(), keys.size() * 4, cudaMemcpyHostToDevice));
  k_search<<<20, 256>>>(dl, (uint32_t)list.size(), dk, (uint32_t)keys.size(), df);
  CK(cudaGetLastError());
  std::vector<uint8_t> found(keys.size());
  CK(cudaMemcpy(found.data(), df, keys.size(), cudaMemcpyDeviceToHost));
  uint64_t search_bad = 0;
  for (size_t i = 0; i < keys.size(); ++i)
    search_bad += (found[i] != 0) != std::binary_search(list.begin(), list.end(), keys[i]);

  const bool ok = views_ok && got[0] == want && got[1] == want && got[2] == want &&
                  legacy == (unsigned)want && fast == want && pair_bad == 0 && search_bad == 0;
  std::printf(
      "{\"scale\": %d, \"ef\": %d, \"seed\": %llu, \"n\": %u, \"dag_edges\": %zu, \"cpu\": %llu, "
      "\"hom_cache\": %zu, \"hom_nocache\": %zu, \"hom_chunked\": %zu, \"legacy_u32\": %u, "
      "\"fast\": %llu, \"c4\": %llu, \"k4\": %llu, \"views_ok\": %s, \"pairs\": %u, "
      "\"pair_mismatches\": %llu, \"search_mismatches\": %llu, \"ok\": %s}\n",
      scale, ef, (unsigned long long)seed, n, dag->idx.size(), (unsigned long long)want, got[0],
      got[1], got[2], legacy, (unsigned long long)fast, (unsigned long long)c4,
      (unsigned long long)k4, views_ok ? "true" : "false", npairs, (unsigned long long)pair_bad,
      (unsigned long long)search_bad, ok ? "true" : "false");
  return ok ? 0 : 1;
}
