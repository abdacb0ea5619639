// Device graph handle: the B200 counterpart of the reference's DeviceGraphCtx
// (include/DeviceGraph.cuh:75-133).  Owns the degree-oriented adjacency in HBM:
//
//   row[v]  uint2 {off4, len}: list of v starts at adj + 4*off4, len ids
//   adj     uint32 ids, every list 16-byte aligned, padded with UINT32_MAX to
//           a multiple of 4 so a list can be read with uint4 loads and staged
//           with cp.async.bulk (16-byte granularity) without bounds fixes
//   wedge[v] uint64: sum of d+(w) over w in N+(v) (per-vertex work estimate)
//
// With relabeling (the default) vertex ids are ranks by (degree, caller id),
// so N+(v) holds only ids > v and the hubs occupy the top id range.
#pragma once
#include <cstdint>
#include <vector>

#include "internal.cuh"

struct gary_count_plan;  // tc.cu: cached tile lists per (pattern, sched)

struct gary_graph {
  int device = 0;
  uint32_t n = 0;
  uint32_t flags = 0;
  uint32_t max_degree = 0;
  uint32_t max_out = 0;
  uint64_t m = 0;          // oriented edges |E+|
  uint64_t adj_words = 0;  // padded length of adj
  uint64_t wedges = 0;
  uint64_t out_deg_sq = 0;
  uint64_t alg_bytes = 0;
  bool relabeled = true;

  gary::DevBuf<uint2> row;
  gary::DevBuf<uint32_t> adj;
  gary::DevBuf<uint64_t> wedge;
  gary::DevBuf<uint32_t> perm;     // rank -> caller id (relabeled only)
  gary::DevBuf<uint64_t> indptr;   // DeviceCSR view: element offsets
  gary::DevBuf<uint32_t> outdeg;   // DeviceCSR view: d+(v)
  gary::DevBuf<uint32_t> coo_row;  // DeviceCOO view, built lazily
  gary::DevBuf<uint32_t> coo_col;

  // symmetric relabeled lists (built lazily for 4-cycle counting)
  gary::DevBuf<uint2> srow;
  gary::DevBuf<uint32_t> sadj;
  uint64_t sadj_words = 0;

  gary_count_plan *plans[8] = {nullptr};
  gary::DevBuf<unsigned long long> result;  // device word for gary_count
  gary_count_stats last{};
  bool last_timed = false;  // ev0/ev1 bracket the last counting kernel
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;

  gary::GraphView view() const { return gary::GraphView{n, row.p, adj.p}; }
  uint64_t device_bytes() const {
    return row.bytes() + adj.bytes() + wedge.bytes() + perm.bytes() + indptr.bytes() +
           outdeg.bytes() + coo_row.bytes() + coo_col.bytes() + srow.bytes() + sadj.bytes();
  }
};

namespace gary {
// Build the symmetric relabeled adjacency (srow/sadj) from the oriented one.
int build_symmetric(gary_graph *g, cudaStream_t s);
void free_plans(gary_graph *g);
}  // namespace gary
