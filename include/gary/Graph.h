// Host graphs and their binary files: the shim of the parts of the reference's
// include/Graph.h that the counting path's callers use (GraphCSR / GraphCOO
// with numV, numE, getDegree, getPtr, getIdx, N; loadFromBinary and
// saveToBinary, Graph.h:157-316), over the library's reader and writer of the
// reference's cereal-archive layout (gary_bin_* in gary_b200.h).
//
//   auto csr = loadFromBinary<GraphCSR>("csr_dag.bin");   // as test/TriQueryTest.cu:51
//   ctx.loadFromHost(std::make_shared<GraphCSR>(std::move(csr)));
//
// Differences: ids are uint32 and offsets uint64 (the file stores int32 /
// int64; equal for ids below 2^31); arrays are plain vectors rather than
// shared_ptr-held ones; errors throw gary::Error.
#pragma once
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "gary/DeviceGraph.cuh"
#include "gary/ops/DeviceIterator.cuh"
#include "gary_b200.h"

class GraphCSR {
 public:
  GraphCSR() = default;
  GraphCSR(std::vector<eidT> ptr, std::vector<vidT> idx) : ptr_(std::move(ptr)), idx_(std::move(idx)) {
    if (ptr_.empty()) ptr_.push_back(0);
    deg_.resize(ptr_.size() - 1);
    for (size_t v = 0; v + 1 < ptr_.size(); ++v) deg_[v] = (vidT)(ptr_[v + 1] - ptr_[v]);
  }
  vidT numV() const { return (vidT)(ptr_.size() - 1); }
  eidT numE() const { return (eidT)idx_.size(); }
  vidT getDegree(vidT v) const { return deg_[v]; }
  const std::vector<vidT> &getDegreeAll() const { return deg_; }
  const std::vector<eidT> &getPtr() const { return ptr_; }
  const std::vector<vidT> &getIdx() const { return idx_; }
  Span<const vidT, void> N(vidT v) const { return Span<const vidT, void>(idx_.data() + ptr_[v], deg_[v]); }

 private:
  std::vector<eidT> ptr_{0};
  std::vector<vidT> idx_;
  std::vector<vidT> deg_;
};

class GraphCOO {
 public:
  GraphCOO() = default;
  GraphCOO(vidT m, std::vector<vidT> row, std::vector<vidT> col)
      : m_(m), row_(std::move(row)), col_(std::move(col)) {}
  vidT numV() const { return m_; }
  eidT numE() const { return (eidT)row_.size(); }
  const std::vector<vidT> &getRow() const { return row_; }
  const std::vector<vidT> &getCol() const { return col_; }

 private:
  vidT m_ = 0;
  std::vector<vidT> row_, col_;
};

template <class GraphT>
GraphT loadFromBinary(const std::string &path);

template <>
inline GraphCSR loadFromBinary<GraphCSR>(const std::string &path) {
  uint32_t fmt = 0, n = 0;
  uint64_t nnz = 0;
  gary::check(gary_bin_info(path.c_str(), &fmt, &n, &nnz), "gary_bin_info");
  std::vector<eidT> ptr((size_t)n + 1);
  std::vector<vidT> idx((size_t)nnz);
  gary::check(gary_bin_read_csr(path.c_str(), ptr.data(), idx.data()), "gary_bin_read_csr");
  return GraphCSR(std::move(ptr), std::move(idx));
}

template <>
inline GraphCOO loadFromBinary<GraphCOO>(const std::string &path) {
  uint32_t fmt = 0, n = 0;
  uint64_t nnz = 0;
  gary::check(gary_bin_info(path.c_str(), &fmt, &n, &nnz), "gary_bin_info");
  std::vector<vidT> row((size_t)nnz), col((size_t)nnz);
  gary::check(gary_bin_read_coo(path.c_str(), row.data(), col.data()), "gary_bin_read_coo");
  return GraphCOO(n, std::move(row), std::move(col));
}

inline void saveToBinary(const GraphCSR &g, const std::string &path) {
  gary::check(gary_bin_write_csr(path.c_str(), g.getPtr().data(), g.getIdx().data(), g.numV(), g.numE()),
              "gary_bin_write_csr");
}
