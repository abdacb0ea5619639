// Views and cooperative iteration for device code: the shim of the reference's
// include/ops/DeviceIterator.cuh:8-426, with the same names (Array, Span,
// IdRange, WorkPartition, interleavedPolicy, chunkedPolicy, warpsPerBlock,
// subGroupId) and the same meaning of every cooperate() form:
//
//   span.cooperate(g)                 each thread of g visits elements rank,
//                                     rank + |g|, ... (lane-strided)
//   range.cooperate<P>(sub, super)    each sub-group of `super` receives whole
//                                     ids; all threads of a sub-group see the
//                                     same sequence.  INTERLEAVED: id i goes
//                                     to sub-group i mod S.  CHUNKED: id i goes
//                                     to sub-group i / ceil(len / S).
//
// One iterator type serves all of them: a position, a step and an end.
// Positions are 64-bit, so edge ranges beyond 2^31 iterate correctly.
// DYNAMIC partitioning is declared but, as in the reference
// (DeviceIterator.cuh:141), not served: the persistent scheduler of the
// library's own counting kernels replaces it.
#pragma once
#include <cooperative_groups.h>

#include <type_traits>

#include "gary/Defines.h"

namespace utils {
using thread_warp =
    cooperative_groups::thread_block_tile<WARP_SIZE, cooperative_groups::thread_block>;
}

static CUDA_INLINE HOST_DEVICE int warpsPerBlock(dim3 blockDim) {
  return (int)(blockDim.x * blockDim.y * blockDim.z / WARP_SIZE);
}

template <typename SubGroup, typename SuperGroup>
static CUDA_INLINE DEVICE_ONLY size_t subGroupId(const SubGroup &sub, const SuperGroup &super) {
  return (size_t)super.thread_rank() / sub.num_threads();
}

enum WorkPartition {
  DYNAMIC = -1,
  INTERLEAVED = 0,
  CHUNKED = 1,
};
static constexpr WorkPartition interleavedPolicy = WorkPartition::INTERLEAVED;
static constexpr WorkPartition chunkedPolicy = WorkPartition::CHUNKED;

// Fixed-size view of N elements (a per-warp shared-memory cache, typically).
template <typename T, size_t N>
struct Array {
  using value_type = T;
  T *data;
  HOST_DEVICE Array(T *d) : data(d) {}
  HOST_DEVICE T &operator[](size_t i) { return data[i]; }
  HOST_DEVICE const T &operator[](size_t i) const { return data[i]; }
  HOST_DEVICE static constexpr size_t size() { return N; }
  HOST_DEVICE T *begin() const { return data; }
  HOST_DEVICE T *end() const { return data + N; }
};

namespace gary_detail {
// Stepping iterator over [pos, end): `*it` is the id itself (Base = void) or
// base[pos].  `it != end` holds while pos < end, so a step past the end stops.
template <typename Id, typename Base>
struct StepIter {
  Id pos, step;
  Base base;
  HOST_DEVICE auto operator*() const {
    if constexpr (std::is_same_v<Base, std::nullptr_t>) return pos;
    else return base[pos];
  }
  HOST_DEVICE StepIter &operator++() {
    pos += step;
    return *this;
  }
  HOST_DEVICE bool operator!=(const StepIter &e) const { return pos < e.pos; }
};

template <typename Id, typename Base>
struct StepRange {
  Id first, last, step;
  Base base;
  HOST_DEVICE StepIter<Id, Base> begin() const { return {first, step, base}; }
  HOST_DEVICE StepIter<Id, Base> end() const { return {last, step, base}; }
};

// the [first, last) share and step of sub-group `sub` in `super`
template <WorkPartition Policy, typename SubGroup, typename SuperGroup>
DEVICE_ONLY CUDA_INLINE void partition(uint64_t lo, uint64_t hi, const SubGroup &sub,
                                       const SuperGroup &super, uint64_t &first, uint64_t &last,
                                       uint64_t &step) {
  static_assert(Policy != DYNAMIC, "DYNAMIC work partitioning is not served");
  const uint64_t id = (uint64_t)super.thread_rank() / sub.num_threads();
  const uint64_t groups = (uint64_t)super.num_threads() / sub.num_threads();
  if (Policy == INTERLEAVED) {
    first = lo + id;
    last = hi;
    step = groups;
  } else {
    const uint64_t chunk = (hi - lo + groups - 1) / groups;
    first = lo + id * chunk;
    last = first + chunk < hi ? first + chunk : hi;
    step = 1;
  }
  if (first > last) first = last;
}
}  // namespace gary_detail

// Contiguous view of `len` elements.  Span<T, void> is a plain view;
// cooperate() turns it into a strided walk for a group of threads.
template <typename T, typename CudaGroup = void>
class Span;

template <typename T>
class Span<T, void> {
 public:
  using value_type = std::remove_cv_t<T>;
  using IterType = T *;
  HOST_DEVICE Span() : ptr_(nullptr), len_(0) {}
  HOST_DEVICE Span(T *ptr, size_t len) noexcept : ptr_(ptr), len_(len) {}
  HOST_DEVICE size_t size() const noexcept { return len_; }
  HOST_DEVICE T *begin() const noexcept { return ptr_; }
  HOST_DEVICE T *end() const noexcept { return ptr_ + len_; }
  HOST_DEVICE T &operator[](size_t i) const noexcept { return ptr_[i]; }

  // lane-strided: thread r of `group` visits elements r, r + |group|, ...
  template <typename CudaGroup>
  DEVICE_ONLY gary_detail::StepRange<uint64_t, T *> cooperate(const CudaGroup &group) const {
    return {(uint64_t)group.thread_rank() < len_ ? (uint64_t)group.thread_rank() : len_, len_,
            (uint64_t)group.num_threads(), ptr_};
  }
  // whole elements per sub-group (every thread of a sub-group sees the same ones)
  template <WorkPartition Policy = interleavedPolicy, typename SubGroup, typename SuperGroup>
  DEVICE_ONLY gary_detail::StepRange<uint64_t, T *> cooperate(const SubGroup &sub,
                                                              const SuperGroup &super) const {
    uint64_t a, b, s;
    gary_detail::partition<Policy>(0, len_, sub, super, a, b, s);
    return {a, b, s, ptr_};
  }

 private:
  T *ptr_;
  size_t len_;
};

// The ids [min, max).
template <typename IdType, typename CudaGroup = void>
class IdRange;

template <typename IdType>
class IdRange<IdType, void> {
 public:
  using value_type = IdType;
  HOST_DEVICE IdRange(IdType lo, IdType hi) : min_(lo), max_(hi) {}
  HOST_DEVICE explicit IdRange(IdType hi) : min_(0), max_(hi) {}
  HOST_DEVICE size_t size() const { return max_ > min_ ? (size_t)(max_ - min_) : 0; }
  HOST_DEVICE gary_detail::StepIter<IdType, std::nullptr_t> begin() const {
    return {min_, 1, nullptr};
  }
  HOST_DEVICE gary_detail::StepIter<IdType, std::nullptr_t> end() const {
    return {max_, 1, nullptr};
  }

  template <typename CudaGroup>
  DEVICE_ONLY gary_detail::StepRange<uint64_t, std::nullptr_t> cooperate(const CudaGroup &g) const {
    const uint64_t lo = (uint64_t)min_, hi = (uint64_t)max_;
    const uint64_t first = lo + g.thread_rank();
    return {first < hi ? first : hi, hi, (uint64_t)g.num_threads(), nullptr};
  }
  template <WorkPartition Policy = interleavedPolicy, typename SubGroup, typename SuperGroup>
  DEVICE_ONLY gary_detail::StepRange<uint64_t, std::nullptr_t> cooperate(
      const SubGroup &sub, const SuperGroup &super) const {
    uint64_t a, b, s;
    gary_detail::partition<Policy>((uint64_t)min_, (uint64_t)max_, sub, super, a, b, s);
    return {a, b, s, nullptr};
  }

 private:
  IdType min_, max_;
};
