// C-ABI glue: error strings, handle lifetime, dispatch of gary_count.
// No C++ exception crosses this boundary: every entry point catches and maps
// to a GARY_ERR_* status (the reference's checkCudaErrors exits the process
// instead, common/HelperCUDA.h:582-595).
#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <iterator>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <unordered_map>
#include <vector>

#include "graph.cuh"
#include "internal.cuh"
#include "mlp.cuh"
#include "patterns.cuh"
#include "tc.cuh"

namespace gary {

namespace {
thread_local char g_error[1024] = {0};
}

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_error, sizeof(g_error), fmt, ap);
  va_end(ap);
}

void clear_error() { g_error[0] = '\0'; }

int device_ordinal() {
  int d = 0;
  cudaGetDevice(&d);
  return d;
}

int sm_count() {
  static int cache[64] = {0};
  int d = device_ordinal();
  if (d >= 0 && d < 64 && cache[d]) return cache[d];
  int v = 0;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d) != cudaSuccess || v <= 0) {
    cudaGetLastError();
    v = 148;
  }
  if (d >= 0 && d < 64) cache[d] = v;
  return v;
}

namespace {
std::mutex g_pool_mu;
cudaMemPool_t g_pools[64] = {};
uint64_t g_pool_keep = ~0ull;  // keep freed scratch mapped, as a caching allocator does
}  // namespace

cudaMemPool_t scratch_pool() {
  const int d = device_ordinal();
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (d < 0 || d >= 64) {
    cudaMemPool_t p = nullptr;
    cudaDeviceGetDefaultMemPool(&p, d);
    return p;
  }
  if (!g_pools[d]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = d;
    if (cudaMemPoolCreate(&g_pools[d], &props) != cudaSuccess) {
      cudaGetLastError();
      cudaDeviceGetDefaultMemPool(&g_pools[d], d);
    } else {
      uint64_t keep = g_pool_keep;
      cudaMemPoolSetAttribute(g_pools[d], cudaMemPoolAttrReleaseThreshold, &keep);
    }
  }
  return g_pools[d];
}

namespace {
struct BlockInfo {
  size_t bytes;
  int dev;
};
std::mutex g_blk_mu;
std::unordered_map<void *, BlockInfo> g_live;      // blocks handed out
std::multimap<size_t, void *> g_cached[64];         // free blocks by rounded size, per device
uint64_t g_cached_bytes[64] = {};

size_t round_block(size_t b) {
  if (b <= (1u << 20)) {
    size_t r = 256;
    while (r < b) r <<= 1;
    return r;
  }
  const size_t step = 2u << 20;
  return (b + step - 1) / step * step;
}

// Returns cached blocks of device d to the driver, largest first, until at
// most keep bytes stay cached.  Caller holds g_blk_mu.
void trim_blocks_locked(int d, uint64_t keep) {
  auto &c = g_cached[d];
  if (c.empty() || g_cached_bytes[d] <= keep) return;
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != d) cudaSetDevice(d);
  while (g_cached_bytes[d] > keep && !c.empty()) {
    auto it = std::prev(c.end());
    cudaFree(it->second);
    g_cached_bytes[d] -= it->first;
    c.erase(it);
  }
  if (cur != d) cudaSetDevice(cur);
}
}  // namespace

cudaError_t persistent_alloc(void **p, size_t bytes) {
  const int d = device_ordinal();
  const size_t rb = round_block(bytes);
  if (d >= 0 && d < 64) {
    std::lock_guard<std::mutex> lk(g_blk_mu);
    auto &c = g_cached[d];
    auto it = c.lower_bound(rb);
    if (it != c.end() && it->first <= rb + rb / 8) {
      *p = it->second;
      g_live[*p] = BlockInfo{it->first, d};
      g_cached_bytes[d] -= it->first;
      c.erase(it);
      return cudaSuccess;
    }
  }
  cudaError_t e = cudaMalloc(p, rb);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    release_cached_memory();
    e = cudaMalloc(p, rb);
  }
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_blk_mu);
  g_live[*p] = BlockInfo{rb, d};
  return cudaSuccess;
}

void persistent_free(void *p) {
  BlockInfo info{0, -1};
  {
    std::lock_guard<std::mutex> lk(g_blk_mu);
    auto it = g_live.find(p);
    if (it != g_live.end()) {
      info = it->second;
      g_live.erase(it);
    }
  }
  if (info.dev < 0 || info.dev >= 64) {
    cudaFree(p);
    return;
  }
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != info.dev) cudaSetDevice(info.dev);
  if (cudaDeviceSynchronize() != cudaSuccess) cudaGetLastError();
  {
    std::lock_guard<std::mutex> lk(g_blk_mu);
    g_cached[info.dev].emplace(info.bytes, p);
    g_cached_bytes[info.dev] += info.bytes;
    uint64_t keep;
    {
      std::lock_guard<std::mutex> lk2(g_pool_mu);
      keep = g_pool_keep;
    }
    trim_blocks_locked(info.dev, keep);
  }
  if (cur != info.dev) cudaSetDevice(cur);
}

void release_cached_memory() {
  {
    std::lock_guard<std::mutex> lk(g_blk_mu);
    for (int d = 0; d < 64; ++d) trim_blocks_locked(d, 0);
  }
  std::lock_guard<std::mutex> lk(g_pool_mu);
  for (int d = 0; d < 64; ++d) {
    if (!g_pools[d]) continue;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != d) cudaSetDevice(d);
    cudaDeviceSynchronize();
    cudaMemPoolTrimTo(g_pools[d], 0);
    if (cur != d) cudaSetDevice(cur);
  }
  cudaGetLastError();
}

void set_pool_keep_bytes(uint64_t bytes) {
  {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    g_pool_keep = bytes;
    for (cudaMemPool_t p : g_pools) {
      if (!p) continue;
      uint64_t keep = bytes;
      cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
      cudaMemPoolTrimTo(p, bytes);
    }
  }
  std::lock_guard<std::mutex> lk(g_blk_mu);
  for (int d = 0; d < 64; ++d) trim_blocks_locked(d, bytes);
}

namespace {
double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
bool trace_on() {
  static const bool on = [] {
    const char *e = std::getenv("GARY_TRACE");
    return e && *e && std::strcmp(e, "0") != 0;
  }();
  return on;
}
}  // namespace

PhaseTrace::PhaseTrace(const char *what_, cudaStream_t s_) : what(what_), s(s_), on(trace_on()) {
  if (on) {
    cudaStreamSynchronize(s);
    t0 = t = now_s();
  }
}

void PhaseTrace::mark(const char *phase) {
  if (!on) return;
  cudaStreamSynchronize(s);
  const double x = now_s();
  std::fprintf(stderr, "[gary trace] %s: %-24s %9.3f ms\n", what, phase, (x - t) * 1e3);
  t = x;
}

PhaseTrace::~PhaseTrace() {
  if (on) std::fprintf(stderr, "[gary trace] %s: %-24s %9.3f ms\n", what, "total", (now_s() - t0) * 1e3);
}

int upload(const uint64_t *ptr, const uint32_t *idx, uint32_t n, uint64_t nnz, uint32_t flags,
           cudaStream_t s, gary_graph **out, const uint64_t *group_off, uint32_t ngroups);
int build_coo(PaddedCSR &c, cudaStream_t s);
int download(gary_graph *g, uint64_t *ptr, uint32_t *idx, uint32_t *perm, cudaStream_t s);

void free_plans(gary_graph *g) {
  for (auto &p : g->plans) {
    delete p;
    p = nullptr;
  }
  delete g->k4_plan;
  delete g->c4_plan;
  g->k4_plan = g->c4_plan = nullptr;
}

namespace {

template <typename F>
int guarded(const char *what, F &&f) {
  clear_error();
  try {
    return f();
  } catch (const std::bad_alloc &) {
    set_error("%s: out of memory", what);
    return GARY_ERR_OOM;
  } catch (const std::exception &e) {
    set_error("%s: %s", what, e.what());
    return GARY_ERR_CUDA;
  } catch (...) {
    set_error("%s: unknown exception", what);
    return GARY_ERR_CUDA;
  }
}

int plan_slot(int pattern, int sched) { return (pattern - 3) * 2 + sched; }

PlanParams g_tuning;  // process-wide knobs of the counting plans (gary_tune)
std::mutex g_tuning_mu;
std::vector<float> g_model;  // process-wide cost model (gary_set_cost_model)
std::mutex g_model_mu;

int count_async(gary_graph *g, int pattern, int sched, cudaStream_t s, unsigned long long *d_out,
                uint32_t shard = 0, uint32_t nshards = 1) {
  GARY_CHECK_ARG(g != nullptr, "graph is NULL");
  GARY_CHECK_ARG(d_out != nullptr, "output pointer is NULL");
  GARY_CHECK_ARG(pattern == GARY_PATTERN_TRIANGLE || pattern == GARY_PATTERN_4CYCLE ||
                     pattern == GARY_PATTERN_4CLIQUE,
                 "unknown pattern %d", pattern);
  GARY_CHECK_ARG(sched == GARY_SCHED_PLAIN || sched == GARY_SCHED_LEARNED, "unknown scheduler %d",
                 sched);
  GARY_CHECK_ARG(nshards >= 1 && shard < nshards, "shard %u of %u is out of range", shard, nshards);
  if (pattern == GARY_PATTERN_4CLIQUE) {
    if (g->dag.max_len > kK4MaxOutDegree) {
      set_error("4-clique counting supports out-degree <= %u (graph has %u)", kK4MaxOutDegree,
                g->dag.max_len);
      return GARY_ERR_UNSUPPORTED;
    }
    if (!g->k4_plan) GARY_TRY(build_k4_plan(g, s, &g->k4_plan));
    return launch_k4(g, g->k4_plan, d_out, s, shard, nshards);
  }
  if (pattern == GARY_PATTERN_4CYCLE) {
    if (!g->c4_plan) GARY_TRY(build_c4_plan(g, s, &g->c4_plan));
    return launch_c4(g, g->c4_plan, d_out, s, shard, nshards);
  }
  const int slot = plan_slot(pattern, sched);
  if (!g->plans[slot]) {
    if (sched == GARY_SCHED_LEARNED) {
      std::vector<float> model;
      {
        std::lock_guard<std::mutex> lk(g_model_mu);
        model = g_model;
      }
      if (model.empty()) {
        set_error("GARY_SCHED_LEARNED needs a cost model: call gary_set_cost_model first");
        return GARY_ERR_INVALID;
      }
      GARY_TRY(build_k3_plan(g, tuned_params(), s, &g->plans[slot], model.data()));
    } else {
      GARY_TRY(build_k3_plan(g, tuned_params(), s, &g->plans[slot]));
    }
  }
  return launch_k3(g, g->plans[slot], d_out, s, shard, nshards);
}

}  // namespace

PlanParams tuned_params() {
  std::lock_guard<std::mutex> lk(g_tuning_mu);
  return g_tuning;
}

// GARY_OK, or the status the error word of a counting launch stands for.
int launch_status(uint32_t err) {
  if (!err) return GARY_OK;
  if (err & kLaunchErrTableFull) {
    set_error("a shared-memory table of the counting kernel overflowed (error word 0x%x): the count "
              "is incomplete", err);
    return GARY_ERR_INTERNAL;
  }
  set_error("a bounded device wait expired (error word 0x%x): the count is incomplete", err);
  return GARY_ERR_TIMEOUT;
}

}  // namespace gary

using gary::guarded;

extern "C" int gary_tune(const char *key, uint64_t value) {
  GARY_CHECK_ARG(key != nullptr, "key is NULL");
  std::lock_guard<std::mutex> lk(gary::g_tuning_mu);
  gary::PlanParams &p = gary::g_tuning;
  const std::string k(key);
  const bool pow2 = value && !(value & (value - 1));
  if (k == "warp_tile_cost") p.warp_tile_cost = value;  // 0: from the work
  else if (k == "cta_tile_cost" && value > 0) p.cta_tile_cost = value;
  else if (k == "warp_cap" && value >= 8 && value <= gary::kWarpTableSlots / 2) p.warp_cap = (uint32_t)value;
  else if (k == "cta_set_words" && (value == 0 || (pow2 && value >= 64 && value <= gary::kTcMaxWarps * gary::kWarpTableSlots)))
    p.cta_set_words = (uint32_t)value;
  else if (k == "stage_wait_polls" && value <= gary::kSpinLimit) p.stage_polls = (uint32_t)value;
  else if (k == "vertex_overhead") p.vertex_overhead = value;
  else if (k == "min_blocks" && (value == 0 || value == 2 || value == 3)) p.min_blocks = (uint32_t)value;
  else if (k == "pool_keep_bytes") gary::set_pool_keep_bytes(value);
  else if (k == "reset") p = gary::PlanParams{};
  else {
    gary::set_error("unknown tuning key '%s' or value %llu out of range", key,
                    (unsigned long long)value);
    return GARY_ERR_INVALID;
  }
  return GARY_OK;
}

extern "C" int gary_set_cost_model(const float *params) {
  std::lock_guard<std::mutex> lk(gary::g_model_mu);
  if (!params) {
    gary::g_model.clear();
    return GARY_OK;
  }
  gary::g_model.assign(params, params + gary::kMlpParams);
  return GARY_OK;
}

extern "C" int gary_tc_features(gary_graph *g, float *d_x, uint8_t *d_legal, void *stream) {
  GARY_CHECK_ARG(g && d_x && d_legal, "NULL argument");
  return guarded("gary_tc_features", [&] {
    cudaStream_t s = gary::as_stream(stream);
    const int slot = gary::plan_slot(GARY_PATTERN_TRIANGLE, GARY_SCHED_PLAIN);
    if (!g->plans[slot]) GARY_TRY(gary::build_k3_plan(g, gary::tuned_params(), s, &g->plans[slot]));
    return gary::k3_features(g, g->plans[slot], d_x, d_legal, s);
  });
}

extern "C" int gary_tc_profile(gary_graph *g, int variant, uint64_t *d_cycles, uint64_t *d_count,
                               void *stream) {
  GARY_CHECK_ARG(g && d_cycles && d_count, "NULL argument");
  GARY_CHECK_ARG(variant >= -1 && variant <= 3, "variant must be -1 (plain) or 0..3");
  return guarded("gary_tc_profile", [&] {
    cudaStream_t s = gary::as_stream(stream);
    const int slot = gary::plan_slot(GARY_PATTERN_TRIANGLE, GARY_SCHED_PLAIN);
    if (!g->plans[slot]) GARY_TRY(gary::build_k3_plan(g, gary::tuned_params(), s, &g->plans[slot]));
    gary::DevBuf<uint8_t> forced;
    if (variant >= 0) {
      GARY_TRY(forced.alloc(g->n, s));
      GARY_CUDA(cudaMemsetAsync(forced.p, variant, g->n, s));
    }
    GARY_CUDA(cudaMemsetAsync(d_cycles, 0, (uint64_t)g->n * 8, s));
    return gary::launch_k3_ctl(g, g->plans[slot], reinterpret_cast<unsigned long long *>(d_count), s,
                               0, 1, variant >= 0 ? forced.p : nullptr,
                               reinterpret_cast<unsigned long long *>(d_cycles));
  });
}

// ---- batches ------------------------------------------------------------
struct gary_exec {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace gary {
namespace {
int batch_count(gary_graph *g, unsigned long long *d_counts, unsigned long long *d_total,
                cudaStream_t s, int sched) {
  GARY_CHECK_ARG(g != nullptr && d_counts != nullptr && d_total != nullptr, "NULL argument");
  GARY_CHECK_ARG(g->ngroups > 0, "graph was not uploaded with gary_batch_upload");
  const int slot = plan_slot(GARY_PATTERN_TRIANGLE, sched);
  if (!g->plans[slot]) GARY_TRY(count_async(g, GARY_PATTERN_TRIANGLE, sched, s, d_total));
  GARY_CUDA(cudaMemsetAsync(d_counts, 0, (uint64_t)g->ngroups * 8, s));
  gary_count_plan *plan = g->plans[slot];
  return launch_k3_ctl(g, plan, d_total, s, 0, 1, plan->variant.p, nullptr, d_counts);
}
}  // namespace
}  // namespace gary

extern "C" int gary_batch_count_async(gary_graph *g, int sched, uint64_t *d_counts, uint64_t *d_total,
                                      void *stream) {
  GARY_CHECK_ARG(sched == GARY_SCHED_PLAIN || sched == GARY_SCHED_LEARNED, "unknown scheduler");
  return guarded("gary_batch_count_async", [&] {
    return gary::batch_count(g, reinterpret_cast<unsigned long long *>(d_counts),
                             reinterpret_cast<unsigned long long *>(d_total), gary::as_stream(stream),
                             sched);
  });
}

extern "C" int gary_batch_capture(gary_graph *g, int sched, uint64_t *d_counts, uint64_t *d_total,
                                  void *stream, gary_exec **out) {
  GARY_CHECK_ARG(out != nullptr, "out is NULL");
  GARY_CHECK_ARG(stream != nullptr, "capture needs a non-default stream");
  return guarded("gary_batch_capture", [&] {
    cudaStream_t s = gary::as_stream(stream);
    // plans are built (allocations, host syncs) before the capture begins
    GARY_TRY(gary::batch_count(g, reinterpret_cast<unsigned long long *>(d_counts),
                               reinterpret_cast<unsigned long long *>(d_total), s, sched));
    GARY_CUDA(cudaStreamSynchronize(s));
    auto e = std::make_unique<gary_exec>();
    GARY_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const int st = gary::batch_count(g, reinterpret_cast<unsigned long long *>(d_counts),
                                     reinterpret_cast<unsigned long long *>(d_total), s, sched);
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(s, &graph);
    if (st != GARY_OK) {
      if (graph) cudaGraphDestroy(graph);
      return st;
    }
    GARY_CUDA(ce);
    e->graph = graph;
    GARY_CUDA(cudaGraphInstantiate(&e->exec, graph, 0));
    *out = e.release();
    return GARY_OK;
  });
}

extern "C" int gary_exec_launch(gary_exec *e, void *stream) {
  GARY_CHECK_ARG(e != nullptr, "exec is NULL");
  GARY_CUDA(cudaGraphLaunch(e->exec, gary::as_stream(stream)));
  return GARY_OK;
}

extern "C" int gary_exec_free(gary_exec *e) {
  if (!e) return GARY_OK;
  if (e->exec) cudaGraphExecDestroy(e->exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  delete e;
  return GARY_OK;
}

extern "C" int gary_graph_drop_plans(gary_graph *g) {
  GARY_CHECK_ARG(g != nullptr, "graph is NULL");
  gary::free_plans(g);
  return GARY_OK;
}

extern "C" const char *gary_last_error(void) { return gary::g_error; }

extern "C" int gary_abi_version(void) { return GARY_ABI_VERSION; }

extern "C" int gary_graph_upload(const uint64_t *ptr, const uint32_t *idx, uint32_t n,
                                 uint64_t nnz, uint32_t flags, void *stream, gary_graph **out) {
  return guarded("gary_graph_upload", [&] {
    return gary::upload(ptr, idx, n, nnz, flags, gary::as_stream(stream), out, nullptr, 0);
  });
}

extern "C" int gary_batch_upload(const uint64_t *group_off, uint32_t ngroups, const uint64_t *ptr,
                                 const uint32_t *idx, uint32_t n, uint64_t nnz, uint32_t flags,
                                 void *stream, gary_graph **out) {
  GARY_CHECK_ARG(group_off != nullptr && ngroups >= 1, "need ngroups >= 1 and host group offsets");
  GARY_CHECK_ARG(!(flags & GARY_KEEP_IDS), "GARY_KEEP_IDS is not supported for batches");
  return guarded("gary_batch_upload", [&] {
    return gary::upload(ptr, idx, n, nnz, flags, gary::as_stream(stream), out, group_off, ngroups);
  });
}

extern "C" int gary_graph_free(gary_graph *g) {
  if (!g) return GARY_OK;
  return guarded("gary_graph_free", [&] {
    gary::free_plans(g);
    if (g->ev0) cudaEventDestroy(g->ev0);
    if (g->ev1) cudaEventDestroy(g->ev1);
    delete g;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      gary::set_error("gary_graph_free: %s", cudaGetErrorString(e));
      return GARY_ERR_CUDA;
    }
    return GARY_OK;
  });
}

extern "C" int gary_graph_get_info(const gary_graph *g, gary_graph_info *out) {
  GARY_CHECK_ARG(g != nullptr && out != nullptr, "NULL argument");
  out->n = g->n;
  out->max_degree = g->max_degree;
  out->max_out_degree = g->dag.max_len;
  out->relabeled = g->keep_ids ? 0u : 1u;
  out->m = g->dag.m;
  out->adj_words = g->dag.words;
  out->wedges = g->wedges;
  out->out_deg_sq = g->out_deg_sq;
  out->alg_bytes = g->alg_bytes;
  out->device_bytes = g->device_bytes();
  return GARY_OK;
}

extern "C" int gary_graph_device_csr(gary_graph *g, gary_device_csr *out) {
  GARY_CHECK_ARG(g != nullptr && out != nullptr, "NULL argument");
  gary::PaddedCSR &c = g->user_view();
  out->m = g->n;
  out->nnz = c.m;
  out->indPtr = c.indptr.p;
  out->colIdx = c.adj.p;
  out->deg = c.outdeg.p;
  return GARY_OK;
}

extern "C" int gary_graph_device_coo(gary_graph *g, gary_device_coo *out) {
  GARY_CHECK_ARG(g != nullptr && out != nullptr, "NULL argument");
  return guarded("gary_graph_device_coo", [&] {
    gary::PaddedCSR &c = g->user_view();
    GARY_TRY(gary::build_coo(c, nullptr));
    out->m = g->n;
    out->nnz = c.m;
    out->rowIdx = c.coo_row.p;
    out->colIdx = c.coo_col.p;
    out->deg = c.outdeg.p;
    return GARY_OK;
  });
}

extern "C" int gary_graph_download(gary_graph *g, uint64_t *ptr, uint32_t *idx, uint32_t *perm) {
  GARY_CHECK_ARG(g != nullptr, "graph is NULL");
  return guarded("gary_graph_download", [&] { return gary::download(g, ptr, idx, perm, nullptr); });
}

extern "C" int gary_count_async(gary_graph *g, int pattern, int sched, void *stream,
                                uint64_t *d_out) {
  return guarded("gary_count_async", [&] {
    return gary::count_async(g, pattern, sched, gary::as_stream(stream),
                             reinterpret_cast<unsigned long long *>(d_out));
  });
}

extern "C" int gary_count(gary_graph *g, int pattern, int sched, void *stream, uint64_t *out) {
  GARY_CHECK_ARG(out != nullptr, "out is NULL");
  GARY_CHECK_ARG(g != nullptr, "graph is NULL");
  return guarded("gary_count", [&] {
    cudaStream_t s = gary::as_stream(stream);
    if (!g->result.p) GARY_TRY(g->result.alloc_persistent(1));
    GARY_TRY(gary::count_async(g, pattern, sched, s, g->result.p));
    unsigned long long h = 0;
    gary::SchedState st{};
    GARY_CUDA(cudaMemcpyAsync(&h, g->result.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    GARY_CUDA(cudaMemcpyAsync(&st, g->last_sched, sizeof(st), cudaMemcpyDeviceToHost, s));
    GARY_CUDA(cudaStreamSynchronize(s));
    GARY_TRY(gary::launch_status(st.error));
    *out = h;
    return GARY_OK;
  });
}

extern "C" int gary_count_shard_async(gary_graph *g, int pattern, int sched, uint32_t shard,
                                      uint32_t nshards, void *stream, uint64_t *d_out) {
  return guarded("gary_count_shard_async", [&] {
    return gary::count_async(g, pattern, sched, gary::as_stream(stream),
                             reinterpret_cast<unsigned long long *>(d_out), shard, nshards);
  });
}

extern "C" int gary_count_status(gary_graph *g, void *stream) {
  GARY_CHECK_ARG(g != nullptr, "graph is NULL");
  GARY_CHECK_ARG(g->last_sched != nullptr, "no count has been launched on this graph");
  return guarded("gary_count_status", [&] {
    cudaStream_t s = gary::as_stream(stream);
    gary::SchedState st{};
    GARY_CUDA(cudaMemcpyAsync(&st, g->last_sched, sizeof(st), cudaMemcpyDeviceToHost, s));
    GARY_CUDA(cudaStreamSynchronize(s));
    return gary::launch_status(st.error);
  });
}

extern "C" int gary_count_last_stats(gary_graph *g, gary_count_stats *out) {
  GARY_CHECK_ARG(g != nullptr && out != nullptr, "NULL argument");
  if (g->last_sched) {
    gary::SchedState st{};
    GARY_CUDA(cudaMemcpy(&st, g->last_sched, sizeof(st), cudaMemcpyDeviceToHost));
    for (int k = 0; k < 4; ++k) g->last.cta_path_tiles[k] = st.cta_path[k];
    g->last.error = st.error;
  }
  if (g->last_span && g->last_span_ctas) {
    // makespan of the launch and the mean time at which its CTAs finished,
    // both from the earliest CTA start
    std::vector<unsigned long long> sp(2ull * g->last_span_ctas);
    GARY_CUDA(cudaMemcpy(sp.data(), g->last_span, sp.size() * 8, cudaMemcpyDeviceToHost));
    unsigned long long t0 = ~0ull, t1 = 0;
    for (uint32_t b = 0; b < g->last_span_ctas; ++b) {
      t0 = std::min(t0, sp[2 * b]);
      t1 = std::max(t1, sp[2 * b + 1]);
    }
    double mean = 0;
    for (uint32_t b = 0; b < g->last_span_ctas; ++b) mean += (double)(sp[2 * b + 1] - t0);
    g->last.makespan_ms = (float)((t1 - t0) * 1e-6);
    g->last.mean_cta_finish_ms = (float)(mean / g->last_span_ctas * 1e-6);
  }
  if (g->last_timed) {
    float ms = 0.f;
    cudaError_t e = cudaEventElapsedTime(&ms, g->ev0, g->ev1);
    if (e == cudaErrorNotReady) {
      cudaGetLastError();
      gary::set_error("the last counting kernel has not finished; synchronise its stream first");
      return GARY_ERR_INVALID;
    }
    if (e != cudaSuccess) {
      gary::set_error("cudaEventElapsedTime: %s", cudaGetErrorString(e));
      cudaGetLastError();
      return GARY_ERR_CUDA;
    }
    g->last.kernel_ms = ms;
  }
  *out = g->last;
  return GARY_OK;
}
