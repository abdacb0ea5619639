// Device graph views and their host owner: the shim of the reference's
// include/DeviceGraph.cuh:15-133 (DeviceCSR, DeviceCOO, DeviceGraph,
// DeviceGraphCtx) on top of the C ABI in gary_b200.h.
//
// What differs from the reference, and why:
//   - The views describe the degree-oriented DAG the library builds on upload
//     (gary_graph_upload): ids are degree ranks unless GARY_KEEP_IDS is given,
//     lists are sorted, start on 32-byte boundaries and are padded with
//     GARY_PAD (UINT32_MAX) up to a multiple of 8.  `deg[v]` is the real
//     length, so N(v) never shows the padding.
//   - The COO view has its own colIdx (the reference aliases the CSR's,
//     DeviceGraph.cuh:117, which the padding would break).
//   - Loading orients the graph.  Given an oriented input (the reference's
//     tests load such a `csr_dag.bin`, test/TriQueryTest.cu:51), a count over
//     the views equals the reference's.  Given a symmetric input, the
//     reference's kernel would count every triangle 6 times (homomorphisms),
//     while the views hold each edge once.
//   - Errors throw gary::Error (a std::runtime_error carrying the GARY_ERR_*
//     status), where the reference throws std::runtime_error /
//     std::invalid_argument (src/DeviceGraph.cu:37-38, 65-66) or exits.
//
// Host code using this header links libgary_b200.so.
#pragma once
#include <cuda_runtime.h>
#include <thrust/tuple.h>

#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "gary/ops/DeviceIterator.cuh"
#include "gary_b200.h"

namespace gary {
class Error : public std::runtime_error {
 public:
  Error(int status, const std::string &what) : std::runtime_error(what), status_(status) {}
  int status() const { return status_; }

 private:
  int status_;
};

inline void check(int status, const char *what) {
  if (status != GARY_OK) throw Error(status, std::string(what) + ": " + gary_last_error());
}
}  // namespace gary

// Non-owning CSR view, passed to kernels by value.
struct DeviceCSR {
  vidT m = 0;
  eidT nnz = 0;
  const eidT *indPtr = nullptr;
  const vidT *colIdx = nullptr;
  const vidT *deg = nullptr;

  using VType = vidT;
  using EType = thrust::tuple<vidT, vidT>;

  HOST_DEVICE vidT numV() const { return m; }
  HOST_DEVICE eidT numE() const { return nnz; }
  HOST_DEVICE vidT getDegree(vidT v) const { return deg[v]; }
  // (v, the eno-th neighbour of v), 0 <= eno < getDegree(v)
  HOST_DEVICE EType getEdge(vidT v, vidT eno) const { return {v, colIdx[indPtr[v] + eno]}; }
  HOST_DEVICE IdRange<vidT, void> V() const { return IdRange<vidT, void>(0, m); }
  HOST_DEVICE Span<const vidT, void> N(vidT v) const {
    return Span<const vidT, void>(colIdx + indPtr[v], deg[v]);
  }
};

// Non-owning COO view: edge e is (rowIdx[e], colIdx[e]), grouped by row.
struct DeviceCOO {
  vidT m = 0;
  eidT nnz = 0;
  const vidT *rowIdx = nullptr;
  const vidT *colIdx = nullptr;
  const vidT *deg = nullptr;

  using VType = vidT;
  using EType = thrust::tuple<vidT, vidT>;

  HOST_DEVICE vidT numV() const { return m; }
  HOST_DEVICE eidT numE() const { return nnz; }
  HOST_DEVICE vidT getDegree(vidT v) const { return deg[v]; }
  HOST_DEVICE EType getEdge(eidT e) const { return {rowIdx[e], colIdx[e]}; }
  HOST_DEVICE IdRange<vidT, void> V() const { return IdRange<vidT, void>(0, m); }
  HOST_DEVICE IdRange<eidT, void> E() const { return IdRange<eidT, void>(0, nnz); }
};

struct DeviceGraph {
  DeviceCSR csr;
  DeviceCOO coo;
};

// Owner of one device graph (a gary_graph handle).  Movable, not copyable.
class DeviceGraphCtx {
 public:
  DeviceGraphCtx() = default;
  // any host CSR type with numV(), numE(), getPtr(), getIdx() (the reference's
  // GraphCSR qualifies, include/Graph.h:157-252)
  template <class HostCSR>
  explicit DeviceGraphCtx(std::shared_ptr<HostCSR> graph, uint32_t flags = GARY_INPUT_DAG) {
    loadFromHost(std::move(graph), flags);
  }
  DeviceGraphCtx(const DeviceGraphCtx &) = delete;
  DeviceGraphCtx &operator=(const DeviceGraphCtx &) = delete;
  DeviceGraphCtx(DeviceGraphCtx &&o) noexcept : g_(std::exchange(o.g_, nullptr)) {}
  DeviceGraphCtx &operator=(DeviceGraphCtx &&o) noexcept {
    if (this != &o) {
      clear();
      g_ = std::exchange(o.g_, nullptr);
    }
    return *this;
  }
  ~DeviceGraphCtx() { clear(); }

  // Replaces the current graph.  flags: GARY_INPUT_DAG (each edge listed once,
  // as the reference's csr_dag.bin) or GARY_INPUT_SYMMETRIC, plus
  // GARY_KEEP_IDS / GARY_VALIDATE.  Mirrors loadFromHost(GraphCSR)
  // (src/DeviceGraph.cu:18-28); the orientation pass runs on the device.
  template <class HostCSR>
  void loadFromHost(std::shared_ptr<HostCSR> graph, uint32_t flags = GARY_INPUT_DAG) {
    if (!graph) throw std::invalid_argument("loadFromHost: null graph");
    const auto &ptr = graph->getPtr();
    const auto &idx = graph->getIdx();
    std::vector<uint64_t> p(ptr.begin(), ptr.end());
    std::vector<uint32_t> i(idx.begin(), idx.end());
    loadFromArrays(p.data(), i.data(), (uint32_t)graph->numV(), (uint64_t)graph->numE(), flags);
  }

  // Host (or, with GARY_INPUT_DEVICE, device) arrays: ptr[n+1], idx[nnz].
  void loadFromArrays(const uint64_t *ptr, const uint32_t *idx, uint32_t n, uint64_t nnz,
                      uint32_t flags = GARY_INPUT_DAG, cudaStream_t stream = nullptr) {
    clear();
    gary::check(gary_graph_upload(ptr, idx, n, nnz, flags, stream, &g_), "gary_graph_upload");
  }

  // Builds the COO view now rather than on first use (src/DeviceGraph.cu:40-47).
  void populateDevice() {
    gary_device_coo coo;
    gary::check(gary_graph_device_coo(handle(), &coo), "gary_graph_device_coo");
  }

  // Releases the device graph (src/DeviceGraph.cu:54-61).
  void clear() {
    if (g_) gary_graph_free(g_);
    g_ = nullptr;
  }

  bool loaded() const { return g_ != nullptr; }

  DeviceCSR getDeviceCSR() {
    gary_device_csr c;
    gary::check(gary_graph_device_csr(handle(), &c), "gary_graph_device_csr");
    return DeviceCSR{c.m, c.nnz, c.indPtr, c.colIdx, c.deg};
  }
  DeviceCOO getDeviceCOO() {
    gary_device_coo c;
    gary::check(gary_graph_device_coo(handle(), &c), "gary_graph_device_coo");
    return DeviceCOO{c.m, c.nnz, c.rowIdx, c.colIdx, c.deg};
  }
  DeviceGraph getDeviceGraph() { return DeviceGraph{getDeviceCSR(), getDeviceCOO()}; }

  gary_graph_info info() const {
    gary_graph_info i;
    gary::check(gary_graph_get_info(handle(), &i), "gary_graph_get_info");
    return i;
  }

  // The oriented lists back on the host, without padding (getHostCSR,
  // src/DeviceGraph.cu:63-81, which copies only m of the m+1 offsets).
  void getHostCSR(std::vector<uint64_t> &ptr, std::vector<uint32_t> &idx) {
    const gary_graph_info i = info();
    ptr.resize((size_t)i.n + 1);
    idx.resize((size_t)i.m);
    gary::check(gary_graph_download(handle(), ptr.data(), idx.data(), nullptr), "gary_graph_download");
  }

  gary_graph *handle() const {
    if (!g_) throw std::logic_error("DeviceGraphCtx: no graph loaded");
    return g_;
  }

 private:
  gary_graph *g_ = nullptr;
};
