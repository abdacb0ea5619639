// Device graph handle: the B200 counterpart of the reference's DeviceGraphCtx
// (include/DeviceGraph.cuh:75-133).  Owns the degree-oriented adjacency in HBM.
//
// A PaddedCSR holds one orientation of the graph:
//   row[v]    uint2 {off4, len}: list of v starts at adj + 4*off4 (32-byte
//             aligned: off4 is even), len ids, padded with UINT32_MAX to a
//             multiple of 8 so a list can be read as whole 32-byte octets
//             (one sector, two uint4 loads) that never reach the next list,
//             and staged with cp.async.bulk (16-byte granularity) without
//             bounds fixes
//   indptr[v] uint64 word offset (= 4*off4) and outdeg[v] = len: the
//             reference's DeviceCSR field layout (DeviceGraph.cuh:15-43)
//
// `dag` is what the kernels read: vertex ids are ranks by (degree, caller
// id), so N+(v) holds only ids > v, every list is in orientation order, and
// the hubs occupy the top id range.  With GARY_KEEP_IDS the same orientation
// is also kept in caller ids (`kept`), which the DeviceCSR / COO views and the
// download return.
#pragma once
#include <cstdint>
#include <vector>

#include "internal.cuh"

struct gary_count_plan;  // tc.cu: cached tile lists per (pattern, sched)

namespace gary {
struct PatternPlan;  // patterns.cu: 4-clique / 4-cycle plans
struct SchedState;   // tc.cuh: scheduler and error words of a counting launch
struct PaddedCSR {
  uint32_t n = 0;
  uint64_t m = 0;      // stored ids
  uint64_t words = 0;  // padded length of adj
  uint32_t max_len = 0;
  DevBuf<uint2> row;
  DevBuf<uint32_t> adj;
  DevBuf<uint64_t> indptr;
  DevBuf<uint32_t> outdeg;
  DevBuf<uint32_t> coo_row;  // COO view, built lazily
  DevBuf<uint32_t> coo_col;
  uint64_t bytes() const {
    return row.bytes() + adj.bytes() + indptr.bytes() + outdeg.bytes() + coo_row.bytes() +
           coo_col.bytes();
  }
};
}  // namespace gary

struct gary_graph {
  int device = 0;
  uint32_t n = 0;
  uint32_t flags = 0;
  uint32_t max_degree = 0;
  uint64_t wedges = 0;
  uint64_t out_deg_sq = 0;
  uint64_t alg_bytes = 0;
  bool keep_ids = false;

  gary::PaddedCSR dag;           // ranked ids: what the kernels read
  gary::PaddedCSR kept;          // caller ids (GARY_KEEP_IDS only)
  gary::DevBuf<uint64_t> wedge;  // per vertex: sum of d+(w) over w in N+(v)
  gary::DevBuf<uint32_t> perm;   // rank -> caller id
  gary::DevBuf<uint32_t> rdeg;   // undirected degree by rank id (cost-model feature)
  // disjoint union of several graphs (gary_batch_upload): graph of each rank id
  uint32_t ngroups = 0;
  std::vector<uint64_t> group_off;
  gary::DevBuf<uint32_t> gid;

  // symmetric ranked lists (built lazily for 4-cycle counting)
  gary::PaddedCSR sym;

  gary_count_plan *plans[8] = {nullptr};
  gary::PatternPlan *k4_plan = nullptr;
  gary::PatternPlan *c4_plan = nullptr;
  gary::DevBuf<unsigned long long> result;  // device word for gary_count
  gary_count_stats last{};
  bool last_timed = false;  // ev0/ev1 bracket the last counting kernel
  const gary::SchedState *last_sched = nullptr;  // scheduler words of the last counting launch
  const unsigned long long *last_span = nullptr;   // triangle launches: per-CTA start / finish ns
  uint32_t last_span_ctas = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;

  gary::GraphView view() const { return gary::GraphView{n, dag.row.p, dag.adj.p, true}; }
  gary::PaddedCSR &user_view() { return keep_ids ? kept : dag; }
  uint64_t device_bytes() const {
    return dag.bytes() + kept.bytes() + sym.bytes() + wedge.bytes() + perm.bytes() + rdeg.bytes() +
           gid.bytes();
  }
};

namespace gary {
void free_plans(gary_graph *g);
// rowid[w] = row owning padded word w of `c`
int padded_rowid(const PaddedCSR &c, DevBuf<uint32_t> &rowid, cudaStream_t s);
// g->sym: both directions of every edge, rank ids, sorted, padded
int build_symmetric(gary_graph *g, cudaStream_t s);
}  // namespace gary
