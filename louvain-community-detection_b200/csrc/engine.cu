// engine.cu -- host side of the B200 Louvain engine: device state, level
// loop, the C ABI (include/louvain_b200.h).
//
// Replaces the reference's host orchestration:
//   main.cu:5-70            run loop and timing            -> lv_run
//   modularity.cu:438-520   modularityOptimization          -> lv_phase_move
//   aggregation.cu:387-462  aggregation                     -> lv_phase_aggregate
//   utils.cu:30-108         allocation, upload, teardown    -> lv_engine_*
// Status codes instead of HANDLE_ERROR's exit() (utils.cuh:95-100).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <new>
#include <string>
#include <system_error>
#include <vector>

#include "../../include/louvain_b200.h"
#include "lv_graph.h"
#include "lv_internal.h"

using namespace lvb;

namespace {

thread_local std::string g_last_error;

lv_status fail(lv_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

lv_status cuda_fail(cudaError_t e, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  cudaGetLastError();  // clear a non-sticky error
  return fail(e == cudaErrorMemoryAllocation ? LV_ERR_NOMEM : LV_ERR_CUDA, m);
}

#define CU(expr)                                          \
  do {                                                    \
    cudaError_t e_ = (expr);                              \
    if (e_ != cudaSuccess) return cuda_fail(e_, #expr);   \
  } while (0)

#define LVTRY(expr)                   \
  do {                                \
    lv_status s_ = (expr);            \
    if (s_ != LV_OK) return s_;       \
  } while (0)

// Device buffers are stream-ordered allocations from the calling engine's
// own memory pool on its stream (set by AllocScope in every entry point), so
// growing a buffer never synchronises the whole device -- several engines
// (the server's lanes) run side by side.  A pool per engine also keeps one
// engine's allocation from reusing a block another engine freed on its
// stream, which would make the first wait for the second's queued work.
// Without a scope: plain cudaMalloc / cudaFree.
thread_local cudaStream_t t_alloc_stream = nullptr;
thread_local cudaMemPool_t t_alloc_pool = nullptr;

struct AllocScope {
  cudaStream_t prev;
  cudaMemPool_t prev_pool;
  explicit AllocScope(const lv_engine* E);
  ~AllocScope() {
    t_alloc_stream = prev;
    t_alloc_pool = prev_pool;
  }
};

// Fault injection for tests (lv_debug_fail_device_alloc): the nth device
// allocation after the hook is set fails as if the device were full.
std::atomic<unsigned long long> g_alloc_count{0};
std::atomic<unsigned long long> g_alloc_fail_at{0};

template <typename T>
cudaError_t dalloc(T** p, size_t count) {
  *p = nullptr;
  const unsigned long long fail_at = g_alloc_fail_at.load(std::memory_order_relaxed);
  if (fail_at && g_alloc_count.fetch_add(1, std::memory_order_relaxed) + 1 == fail_at)
    return cudaErrorMemoryAllocation;
  if (count == 0) count = 1;
  if (t_alloc_stream && t_alloc_pool)
    return cudaMallocFromPoolAsync((void**)p, count * sizeof(T), t_alloc_pool, t_alloc_stream);
  if (t_alloc_stream) return cudaMallocAsync((void**)p, count * sizeof(T), t_alloc_stream);
  return cudaMalloc((void**)p, count * sizeof(T));
}

template <typename T>
void dfree(T*& p) {
  if (p) {
    if (t_alloc_stream) cudaFreeAsync((void*)p, t_alloc_stream);
    else cudaFree((void*)p);
  }
  p = nullptr;
}

// Hub plan totals, written after the class counts (cls_count[0..8]) so one
// copy brings both to the host: [10] dispatch chunks, [11] move units,
// [12..13] staged entries (u64), [14..15] chunk-table words (u64).
constexpr int kHubTotals = 10;

// The hub plan of a level on the device (one block).  For every hub
// (class 8 of the degree partition, order[hs .. hs + hc)): its dispatch
// chunks of kHubChunk entries, its hash partitions (move units: about
// kHubPartKeys distinct communities each, at most kHubMaxParts), and its
// offsets in the staging copy and the chunk table, all as exclusive scans
// over the hubs.  `cap` is the capacity of the per-hub arrays; a level
// with more hubs writes no plan and leaves the totals at ~0 (the host
// reports it).
__global__ void __launch_bounds__(1024)
    hub_plan_kernel(const uint64_t* __restrict__ off, const uint32_t* __restrict__ order,
                    uint32_t* cls_count, uint32_t n, uint32_t cap, uint32_t* chunk_start,
                    uint32_t* unit_start, uint32_t* nparts, uint64_t* stage_off,
                    uint64_t* ct_off) {
  __shared__ unsigned long long sh[33];
  uint32_t hs = 0;
  for (int c = 0; c < 8; c++) hs += cls_count[c];
  const uint32_t hc = cls_count[8];
  uint64_t* tot64 = reinterpret_cast<uint64_t*>(cls_count + 12);
  if (hc > cap) {
    if (threadIdx.x == 0) {
      cls_count[kHubTotals] = cls_count[kHubTotals + 1] = ~0u;
      tot64[0] = tot64[1] = ~0ull;
    }
    return;
  }
  unsigned long long c_chunks = 0, c_units = 0, c_stage = 0, c_ct = 0, t;
  for (uint32_t base = 0; base < hc; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    unsigned long long d = 0, nch = 0, np = 0;
    if (i < hc) {
      const uint32_t v = order[hs + i];
      d = off[v + 1] - off[v];
      nch = (d + kHubChunk - 1) / kHubChunk;
      const unsigned long long distinct = d < n ? d : n;
      np = (distinct + kHubPartKeys - 1) / kHubPartKeys;
      np = np < 1 ? 1 : (np > kHubMaxParts ? kHubMaxParts : np);
    }
    const unsigned long long ct = nch * (np + 1);
    const unsigned long long x_ch = block_exclusive_scan(nch, sh, &t);
    const unsigned long long s_ch = c_chunks;
    c_chunks += t;
    const unsigned long long x_u = block_exclusive_scan(np, sh, &t);
    const unsigned long long s_u = c_units;
    c_units += t;
    const unsigned long long x_st = block_exclusive_scan(d, sh, &t);
    const unsigned long long s_st = c_stage;
    c_stage += t;
    const unsigned long long x_ct = block_exclusive_scan(ct, sh, &t);
    const unsigned long long s_ct = c_ct;
    c_ct += t;
    if (i < hc) {
      chunk_start[i] = (uint32_t)(s_ch + x_ch);
      unit_start[i] = (uint32_t)(s_u + x_u);
      nparts[i] = (uint32_t)np;
      stage_off[i] = s_st + x_st;
      ct_off[i] = s_ct + x_ct;
    }
  }
  if (threadIdx.x == 0) {
    chunk_start[hc] = (uint32_t)c_chunks;
    unit_start[hc] = (uint32_t)c_units;
    cls_count[kHubTotals] = (uint32_t)c_chunks;
    cls_count[kHubTotals + 1] = (uint32_t)c_units;
    tot64[0] = c_stage;
    tot64[1] = c_ct;
  }
}

// The hub plan's maps (a warp per hub): dispatch chunk -> (hub, chunk) in
// hub_map[0 .. hb) and hub_map[hb .. 2 hb); move unit -> (hub, partition,
// partitions of the hub).
__global__ void hub_fill_kernel(uint32_t hc, uint32_t hb, const uint32_t* __restrict__ chunk_start,
                                const uint32_t* __restrict__ unit_start,
                                const uint32_t* __restrict__ nparts, uint32_t* hub_map,
                                uint32_t* unit_hub, uint32_t* unit_part, uint32_t* unit_np) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < hc; i += warps) {
    const uint32_t c0 = chunk_start[i], c1 = chunk_start[i + 1];
    for (uint32_t j = c0 + lane; j < c1; j += 32) {
      hub_map[j] = i;
      hub_map[hb + j] = j - c0;
    }
    const uint32_t u0 = unit_start[i], np = nparts[i];
    for (uint32_t p = lane; p < np; p += 32) {
      unit_hub[u0 + p] = i;
      unit_part[u0 + p] = p;
      unit_np[u0 + p] = np;
    }
  }
}

// Sum of degrees per move class (only for the byte counts of profiling).
__global__ void class_degree_kernel(const uint64_t* off, uint32_t n,
                                    unsigned long long* out) {
  __shared__ unsigned long long s[kClasses];
  if (threadIdx.x < kClasses) s[threadIdx.x] = 0ull;
  __syncthreads();
  unsigned long long local[kClasses] = {};  // per thread, then per warp
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += gridDim.x * blockDim.x) {
    const uint64_t d = off[v + 1] - off[v];
    const int c = move_class_of_degree(d);
#pragma unroll
    for (int k = 0; k < kClasses; k++) local[k] += (k == c) ? d : 0ull;
  }
#pragma unroll
  for (int k = 0; k < kClasses; k++) {
    unsigned long long x = local[k];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0 && x) atomicAdd(&s[k], x);
  }
  __syncthreads();
  if (threadIdx.x < kClasses) atomicAdd(&out[threadIdx.x], s[threadIdx.x]);
}

// Timed launch groups.
enum KId {
  K_MOVE1 = 0,  // .. K_MOVE1 + 6 = bucket 7's shared-table class
  K_HUB = 7,    // bucket 7's multi-block class (degree > 2048)
  K_APPLY = 8,
  K_MODULARITY = 9,
  K_LEVEL_INIT = 10,
  K_CONTRACT = 11,
  K_COUNT = 12
};
const char* kKName[K_COUNT] = {"move_b1", "move_b2", "move_b3",    "move_b4",
                               "move_b5", "move_b6", "move_b7",    "move_hub",
                               "apply",   "modularity", "level_init", "contract"};

struct KStat {
  uint64_t launches = 0;
  double ms = 0.0;
  double bytes = 0.0;
};

struct PendingTiming {
  int id;
  cudaEvent_t a, b;
  double bytes;
};

}  // namespace

void lvb_set_error(const std::string& msg) { g_last_error = msg; }
// graph_io.cpp: a Matrix Market file's edge lines (0-based, validated).
lv_status lvb_parse_mtx(const char* path, uint32_t* n_out, std::vector<uint32_t>& src,
                        std::vector<uint32_t>& dst, std::vector<float>& ws);

// Opt-in host-side trace (LVB200_TRACE=1): wall-clock time of each step of
// the level loop on stderr.
namespace {
struct Trace {
  bool on;
  std::chrono::steady_clock::time_point t0;
  Trace() : on(getenv("LVB200_TRACE") != nullptr), t0(std::chrono::steady_clock::now()) {}
  void mark(const char* what, uint32_t level, uint32_t n) {
    if (!on) return;
    const auto t = std::chrono::steady_clock::now();
    static std::atomic<int> next_id{0};
    thread_local int id = next_id++;
    fprintf(stderr, "[lvb200] t%d level=%u V=%u %-28s %9.3f ms\n", id, level, n, what,
            std::chrono::duration<double, std::milli>(t - t0).count());
    t0 = t;
  }
  void reset() { t0 = std::chrono::steady_clock::now(); }
};
thread_local Trace g_trace;  // per thread: server lanes step concurrently
}  // namespace

namespace lvb {
static std::atomic<unsigned long long> g_launches{0};
// Launches recorded while a stream is captured only tally the graph's
// kernels (t_tally); the graph's launches count them when it runs.
thread_local bool t_capturing = false;
thread_local unsigned long long t_tally = 0;
void count_launches(unsigned k) {
  if (t_capturing) {
    t_tally += k;
    return;
  }
  g_launches.fetch_add(k, std::memory_order_relaxed);
}
unsigned long long launch_count() { return g_launches.load(std::memory_order_relaxed); }
static std::atomic<unsigned long long> g_syncs{0};
cudaError_t counted_sync(cudaStream_t st) {
  g_syncs.fetch_add(1, std::memory_order_relaxed);
  return cudaStreamSynchronize(st);
}
unsigned long long sync_count() { return g_syncs.load(std::memory_order_relaxed); }
}  // namespace lvb

struct lv_engine {
  lv_config cfg;
  cudaStream_t st = nullptr;
  bool own_stream = false;
  cudaMemPool_t pool = nullptr;  // this engine's stream-ordered allocations
  int device = 0;

  // capacities of the allocations below
  uint32_t cap_n = 0;
  uint64_t cap_e = 0;

  // level-0 CSR: engine copy or caller device buffers
  uint64_t* in_off = nullptr;
  uint32_t* in_col = nullptr;
  float* in_w = nullptr;
  bool in_owned = false;
  uint64_t* own_off = nullptr;
  uint32_t* own_col = nullptr;
  float* own_w = nullptr;

  // contracted levels, ping-pong
  uint64_t* c_off[2] = {nullptr, nullptr};
  uint32_t* c_col[2] = {nullptr, nullptr};
  float* c_w[2] = {nullptr, nullptr};
  int cur = -1;  // -1: level 0 reads the input CSR

  // per-vertex state
  float* k = nullptr;
  uint32_t* comm = nullptr;
  uint32_t* comm_sz = nullptr;
  double* tot = nullptr;
  // second copy of the community state (fused bucket steps, StepIO)
  uint32_t* comm_alt = nullptr;
  uint32_t* sz_alt = nullptr;
  double* tot_alt = nullptr;
  uint32_t* comm_start = nullptr;  // communities when the pass began (single graph)
  uint32_t* order = nullptr;
  uint32_t* prop = nullptr;
  uint32_t* cls_count = nullptr;
  uint32_t* assignment = nullptr;  // [n0]
  uint32_t* part_tmp = nullptr;
  LevelScalars* sc = nullptr;
  LevelScalars* sc_host = nullptr;  // pinned
  uint32_t* h_counts = nullptr;     // pinned [16]

  double* partials = nullptr;
  size_t partials_cap = 0;
  uint32_t* hub_map = nullptr;  // [blk_vertex | blk_chunk] for dispatch
  size_t hub_map_cap = 0;
  HubArena hub;
  size_t hub_count_cap = 0, hub_blocks_cap = 0, hub_units_cap = 0;
  size_t hub_stage_cap = 0, hub_ct_cap = 0;
  uint32_t* hub_chunk_start = nullptr;  // [hub cap + 1] first dispatch chunk per hub

  ContractBuffers cb{};
  ScanScratch scan;
  SortBuffers sb{};             // contraction by sorting (on demand)
  unsigned char* sb_scan = nullptr;

  // current level
  uint32_t n0 = 0;
  uint32_t n = 0;
  uint64_t e = 0;
  bool loaded = false;
  bool level_ready = false;
  bool finished = false;
  // The level's communities count as moves of the assignment (the
  // reference's graphVertToComm, modularity.cu:515-517) when the move phase
  // returned true or a caller set them; `assignment` itself holds the
  // level-start map and is composed once per level, at aggregation.
  bool accepted = false;
  DispatchPlan plan{};
  double q_last = 0.0;
  std::vector<lv_level_info> levels;

  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // A single graph's contraction leaves its entry count, error flag and
  // time to be read at the next synchronisation (the next level's class
  // counts), so a level boundary costs no extra host round trip.
  bool agg_pending = false;
  cudaEvent_t agg_ev0 = nullptr, agg_ev1 = nullptr;
  uint64_t* h_pending = nullptr;  // pinned: the deferred entry count
  // the contraction's front was launched behind the level graph and its
  // class sizes read with the level's result (whole-run loop only)
  bool front_ready = false;

  // kernel timing
  bool profiling = false;
  KStat kst[K_COUNT];
  std::vector<cudaEvent_t> ev_free;
  std::vector<PendingTiming> pending;
  // batched form: the level holds n_graphs graphs (block-diagonal union)
  bool batch = false;
  uint32_t n_graphs = 0;
  GraphState* gs = nullptr;       // [graph cap] device
  GraphState* gs_host = nullptr;  // [graph cap] pinned
  uint32_t* gid = nullptr;        // [cap_n] graph of every level vertex
  uint32_t* goff_dev = nullptr;   // [graph cap + 1] level vertex offsets
  uint32_t* graph0 = nullptr;     // [n0] input graph of every input vertex
  uint32_t* gbase = nullptr;      // [graph cap] finalisation bases
  uint32_t* gdrop = nullptr;      // [graph cap] graphs dropped at contraction
  size_t graph_cap = 0;
  uint32_t* batch_out = nullptr;  // local assignment of lv_batch_run
  size_t batch_out_cap = 0;
  // per-pass lists of the vertices of graphs still moving (classes 1..7;
  // class 8 copied once per level), their lengths, and the runs' places
  uint32_t* act_order = nullptr;
  size_t act_order_cap = 0;
  uint32_t* act_cnt = nullptr;  // [16]
  uint32_t* cg = nullptr;       // [kMoveClasses * (graph cap + 1)]
  uint32_t* cg_new = nullptr;

  // all passes of a level as one graph (WHILE node), one per key (form,
  // rule, tuning, which kernel classes are non-empty), most recent last
  struct LevelExec {
    uint64_t key;
    cudaGraphExec_t exec;
    unsigned long long launches;  // kernels per pass
  };
  std::vector<LevelExec> level_execs;
  // one pass of the current level captured as a CUDA graph (timing mode)
  cudaGraphExec_t pass_exec = nullptr;
  bool capturing = false;
  std::vector<PendingTiming> graph_timings;  // event pairs inside the graph
  unsigned long long pass_launches = 0;      // kernels per replay (timing mode)
  unsigned long long level_launches = 0;     // kernels per pass of the level graph
  unsigned long long* d_class_deg = nullptr;
  uint64_t class_deg[kClasses] = {};
  // move kernel variant of every bucket (1..7): defaults or lv_autotune's pick
  // the pass descriptor (device); the level graphs built on it are kept
  // across levels and runs
  PassDesc* d_desc = nullptr;
  // persistent level kernel: barrier / timer state (device) and its pinned
  // host mirror
  LevelLoopState* loop_state = nullptr;
  PassDesc* desc_host = nullptr;   // pinned staging of the descriptor
  cudaEvent_t desc_ev = nullptr;   // its last copy
  LevelLoopState* loop_host = nullptr;
  uint8_t tune[8] = {kDefaultVariant[0], kDefaultVariant[1], kDefaultVariant[2],
                     kDefaultVariant[3], kDefaultVariant[4], kDefaultVariant[5],
                     kDefaultVariant[6], kDefaultVariant[7]};

  const uint64_t* off() const { return cur < 0 ? in_off : c_off[cur]; }
  const uint32_t* col() const { return cur < 0 ? in_col : c_col[cur]; }
  const float* wts() const { return cur < 0 ? in_w : c_w[cur]; }

  LevelView view() const {
    LevelView L;
    L.n = n;
    L.off = off();
    L.col = col();
    L.w = wts();
    L.k = k;
    L.comm = comm;
    L.comm_sz = comm_sz;
    L.tot = tot;
    L.comm_alt = comm_alt;
    L.sz_alt = sz_alt;
    L.tot_alt = tot_alt;
    L.sc = sc;
    L.gid = batch ? gid : nullptr;
    L.gs = batch ? gs : nullptr;
    L.n_graphs = batch ? n_graphs : 0u;
    return L;
  }
};

namespace {

AllocScope::AllocScope(const lv_engine* E) : prev(t_alloc_stream), prev_pool(t_alloc_pool) {
  t_alloc_stream = E ? E->st : nullptr;
  t_alloc_pool = E ? E->pool : nullptr;
}

cudaEvent_t take_event(lv_engine* E) {
  if (!E->ev_free.empty()) {
    cudaEvent_t e = E->ev_free.back();
    E->ev_free.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Records an event; inside a stream capture it becomes an external event
// node of the graph, so every replay re-records it.
void record_event(lv_engine* E, cudaEvent_t ev) {
  if (E->capturing)
    cudaEventRecordWithFlags(ev, E->st, cudaEventRecordExternal);
  else
    cudaEventRecord(ev, E->st);
}

// Opens a timed launch group; returns the start event (nullptr when off).
cudaEvent_t prof_begin(lv_engine* E) {
  if (!E->profiling) return nullptr;
  cudaEvent_t a = take_event(E);
  record_event(E, a);
  return a;
}

void prof_end(lv_engine* E, cudaEvent_t a, int id, double bytes) {
  if (!a) return;
  cudaEvent_t b = take_event(E);
  record_event(E, b);
  E->pending.push_back(PendingTiming{id, a, b, bytes});
}

// Accumulates the timings of the last replay of the pass graph.
void prof_collect_graph(lv_engine* E) {
  for (const PendingTiming& p : E->graph_timings) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
      E->kst[p.id].launches++;
      E->kst[p.id].ms += ms;
      E->kst[p.id].bytes += p.bytes;
    }
  }
  cudaGetLastError();
}

// Drops the per-level pass graph of the timing mode (the level graph of
// the WHILE loop is kept: it reads the level from the descriptor).
void drop_pass_graph(lv_engine* E) {
  if (E->pass_exec) cudaGraphExecDestroy(E->pass_exec);
  E->pass_exec = nullptr;
  for (const PendingTiming& p : E->graph_timings) {
    E->ev_free.push_back(p.a);
    E->ev_free.push_back(p.b);
  }
  E->graph_timings.clear();
  E->pass_launches = 0;
}

// Folds the finished groups into the totals (call after a stream sync).
void prof_collect(lv_engine* E) {
  for (const PendingTiming& p : E->pending) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
      E->kst[p.id].launches++;
      E->kst[p.id].ms += ms;
      E->kst[p.id].bytes += p.bytes;
    }
    E->ev_free.push_back(p.a);
    E->ev_free.push_back(p.b);
  }
  E->pending.clear();
  cudaGetLastError();
}

void free_state(lv_engine* E) {
  dfree(E->own_off);
  dfree(E->own_col);
  dfree(E->own_w);
  for (int i = 0; i < 2; i++) {
    dfree(E->c_off[i]);
    dfree(E->c_col[i]);
    dfree(E->c_w[i]);
  }
  dfree(E->k);
  dfree(E->comm);
  dfree(E->comm_sz);
  dfree(E->tot);
  dfree(E->comm_alt);
  dfree(E->sz_alt);
  dfree(E->tot_alt);
  dfree(E->comm_start);
  dfree(E->order);
  dfree(E->prop);
  dfree(E->cls_count);
  dfree(E->assignment);
  dfree(E->gid);
  dfree(E->graph0);
  dfree(E->part_tmp);
  dfree(E->partials);
  dfree(E->hub_map);
  dfree(E->hub.best);
  dfree(E->hub.own);
  dfree(E->hub.hot);
  dfree(E->hub.hot_any);
  dfree(E->hub.nparts);
  dfree(E->hub.stage_off);
  dfree(E->hub.ct_off);
  dfree(E->hub.stage);
  dfree(E->hub.ct);
  dfree(E->hub.blk_vertex);
  dfree(E->hub.blk_chunk);
  dfree(E->hub.blk_nchunks);
  dfree(E->hub.unit_g);
  dfree(E->hub.unit_c);
  dfree(E->hub.unit_start);
  dfree(E->hub_chunk_start);
  ContractBuffers& B = E->cb;
  dfree(B.flag_id);
  dfree(B.mem_off);
  dfree(B.cursor);
  dfree(B.members);
  dfree(B.cnew);
  dfree(B.mstart);
  dfree(B.comm_list);
  dfree(B.comm_cls);
  dfree(B.comm_deg);
  dfree(B.seg);
  dfree(B.new_deg);
  dfree(B.tcol);
  dfree(B.tw);
  dfree(B.tmp);
  dfree(B.counts);
  dfree(B.keys);
  dfree(B.vals);
  dfree(B.g_tab_off);
  dfree(B.g_tab_size);
  dfree(B.g_blk_comm);
  dfree(B.g_blk_chunk);
  dfree(B.g_blk_first);
  B.table_cap = 0;
  B.g_cap = 0;
  if (E->scan.buf) cudaFree(E->scan.buf);
  E->scan.buf = nullptr;
  E->scan.bytes = 0;
  E->sb.cap = 0;
  dfree(E->sb.keys[0]);
  dfree(E->sb.keys[1]);
  dfree(E->sb.vals[0]);
  dfree(E->sb.vals[1]);
  dfree(E->sb.pos);
  dfree(E->sb.counts);
  dfree(E->sb_scan);
  E->sb.scan.buf = nullptr;
  E->sb.scan.bytes = 0;
  E->partials_cap = E->hub_map_cap = 0;
  E->hub_count_cap = E->hub_blocks_cap = E->hub_units_cap = 0;
  E->hub_stage_cap = E->hub_ct_cap = 0;
  E->cap_n = 0;
  E->cap_e = 0;
  E->in_off = nullptr;
  E->in_col = nullptr;
  E->in_w = nullptr;
}

cudaError_t grow_tables(void* ctx, size_t slots, size_t entries) {
  lv_engine* E = static_cast<lv_engine*>(ctx);
  ContractBuffers& B = E->cb;
  // a capacity is zeroed before its buffers are freed, so a failed
  // allocation never leaves a freed buffer behind a stale capacity
  if (slots > B.table_cap) {
    B.table_cap = 0;
    dfree(B.keys);
    dfree(B.vals);
    size_t cap = std::max<size_t>(slots, 1 << 16);
    cudaError_t e = dalloc(&B.keys, cap);
    if (e != cudaSuccess) return e;
    e = dalloc(&B.vals, cap);
    if (e != cudaSuccess) return e;
    B.table_cap = cap;
  }
  if (entries > B.g_cap) {
    B.g_cap = 0;
    dfree(B.g_tab_off);
    dfree(B.g_tab_size);
    dfree(B.g_blk_comm);
    dfree(B.g_blk_chunk);
    dfree(B.g_blk_first);
    size_t cap = std::max<size_t>(entries, 1024);
    cudaError_t e = dalloc(&B.g_tab_off, cap);
    if (e != cudaSuccess) return e;
    e = dalloc(&B.g_tab_size, cap);
    if (e != cudaSuccess) return e;
    e = dalloc(&B.g_blk_comm, cap);
    if (e != cudaSuccess) return e;
    e = dalloc(&B.g_blk_chunk, 2 * cap);
    if (e != cudaSuccess) return e;
    e = dalloc(&B.g_blk_first, cap + 1);
    if (e != cudaSuccess) return e;
    B.g_cap = cap;
  }
  return cudaSuccess;
}

lv_status ensure_capacity(lv_engine* E, uint32_t n, uint64_t e, bool need_input) {
  if (n <= E->cap_n && e <= E->cap_e && (!need_input || E->own_off)) return LV_OK;
  free_state(E);
  const size_t N = n, N1 = (size_t)n + 1, EE = e;
  CU(dalloc(&E->k, N));
  CU(dalloc(&E->comm, N));
  CU(dalloc(&E->comm_sz, N));
  CU(dalloc(&E->tot, N));
  CU(dalloc(&E->comm_alt, N));
  CU(dalloc(&E->sz_alt, N));
  CU(dalloc(&E->tot_alt, N));
  CU(dalloc(&E->comm_start, N));
  CU(dalloc(&E->order, N));
  CU(dalloc(&E->prop, N));
  CU(dalloc(&E->cls_count, 16));
  CU(dalloc(&E->assignment, N));
  CU(dalloc(&E->gid, N));
  CU(dalloc(&E->graph0, N));
  const size_t ptw = partition_tmp_words(N) + 64;
  CU(dalloc(&E->part_tmp, ptw));
  for (int i = 0; i < 2; i++) {
    CU(dalloc(&E->c_off[i], N1));
    CU(dalloc(&E->c_col[i], EE));
    CU(dalloc(&E->c_w[i], EE));
  }
  if (need_input) {
    CU(dalloc(&E->own_off, N1));
    CU(dalloc(&E->own_col, EE));
    CU(dalloc(&E->own_w, EE));
  }
  ContractBuffers& B = E->cb;
  CU(dalloc(&B.flag_id, N));
  CU(dalloc(&B.mem_off, N));
  CU(dalloc(&B.cursor, N));
  CU(dalloc(&B.members, N));
  CU(dalloc(&B.cnew, N));
  CU(dalloc(&B.mstart, N1));
  CU(dalloc(&B.comm_list, N));
  CU(dalloc(&B.comm_cls, N));
  CU(dalloc(&B.comm_deg, N));
  CU(dalloc(&B.seg, N));
  CU(dalloc(&B.new_deg, N1));
  CU(dalloc(&B.tcol, EE));
  CU(dalloc(&B.tw, EE));
  CU(dalloc(&B.tmp, ptw));
  CU(dalloc(&B.counts, 16));
  B.host_counts = E->h_counts + 16;
  B.table_cap = 0;
  B.g_cap = 0;
  const size_t scan_cap = std::max<size_t>(N1, partition_tmp_words(N)) + 1024;
  E->scan.bytes = scan_scratch_bytes(scan_cap);
  CU(cudaMalloc(&E->scan.buf, E->scan.bytes));
  E->cap_n = n;
  E->cap_e = e;
  return LV_OK;
}

lv_status check_device_error(lv_engine* E);

// The reads a deferred contraction left (after a synchronisation that
// covered h_pending and sc_host): the entry count, the contraction's time,
// the device error flag.
lv_status finish_pending(lv_engine* E) {
  if (!E->agg_pending) return LV_OK;
  E->agg_pending = false;
  E->e = E->h_pending[0];
  float ms = 0.0f;
  if (cudaEventElapsedTime(&ms, E->agg_ev0, E->agg_ev1) == cudaSuccess && !E->levels.empty())
    E->levels.back().aggregate_ms = ms;
  cudaGetLastError();
  return check_device_error(E);
}

// Completes a deferred contraction's reads now (entry points that look at
// the level outside the level loop).
lv_status resolve_pending(lv_engine* E) {
  if (!E || !E->agg_pending) return LV_OK;
  CU(cudaMemcpyAsync(E->h_pending, E->cb.counts + 8, sizeof(uint64_t), cudaMemcpyDeviceToHost,
                     E->st));
  CU(cudaMemcpyAsync(E->sc_host, E->sc, sizeof(LevelScalars), cudaMemcpyDeviceToHost, E->st));
  CU(counted_sync(E->st));
  return finish_pending(E);
}

// Degree classes, work plan, hub tables for the current level.
lv_status prepare_level(lv_engine* E, bool sync_scalars = true) {
  const uint32_t n = E->n;
  cudaStream_t st = E->st;
  drop_pass_graph(E);
  CU(partition_by_degree(E->off(), n, E->order, E->cls_count, E->part_tmp,
                         E->scan, st));
  // The hub plan is built on the device and its totals ride on the class
  // counts' copy.  Its per-hub arrays are sized for the most hubs the level
  // can hold: a hub has more than kHubSmemMaxDeg entries, and E->e (the
  // previous level's entry count while a contraction's reads are pending)
  // bounds the level's entries.  A level with more hubs than that (a union
  // that gained graphs) plans again after the copy.
  HubArena& H = E->hub;
  auto plan_hubs = [&](uint64_t cap) -> lv_status {
    if (cap > E->hub_count_cap) {
      E->hub_count_cap = 0;  // zeroed before the frees (see grow_tables)
      dfree(E->hub_chunk_start);
      dfree(H.best);
      dfree(H.own);
      dfree(H.hot);
      dfree(H.hot_any);
      dfree(H.nparts);
      dfree(H.stage_off);
      dfree(H.ct_off);
      dfree(H.unit_start);
      CU(dalloc(&E->hub_chunk_start, (size_t)cap + 1));
      CU(dalloc(&H.unit_start, (size_t)cap + 1));
      CU(dalloc(&H.best, cap));
      CU(dalloc(&H.own, cap));
      CU(dalloc(&H.hot, cap));
      CU(dalloc(&H.hot_any, cap));
      CU(dalloc(&H.nparts, cap));
      CU(dalloc(&H.stage_off, cap));
      CU(dalloc(&H.ct_off, cap));
      E->hub_count_cap = cap;
    }
    (count_launches(1), hub_plan_kernel<<<1, 1024, 0, st>>>(
        E->off(), E->order, E->cls_count, n, (uint32_t)E->hub_count_cap, E->hub_chunk_start,
        H.unit_start, H.nparts, H.stage_off, H.ct_off));
    CU(cudaGetLastError());
    return LV_OK;
  };
  const uint64_t hub_bound = std::min<uint64_t>(n, E->e / (kHubSmemMaxDeg + 1));
  if (hub_bound) LVTRY(plan_hubs(hub_bound));
  CU(cudaMemcpyAsync(E->h_counts, E->cls_count, 16 * sizeof(uint32_t),
                     cudaMemcpyDeviceToHost, st));
  if (E->agg_pending) {  // the previous contraction's reads ride on this sync
    CU(cudaMemcpyAsync(E->h_pending, E->cb.counts + 8, sizeof(uint64_t), cudaMemcpyDeviceToHost,
                       st));
    CU(cudaMemcpyAsync(E->sc_host, E->sc, sizeof(LevelScalars), cudaMemcpyDeviceToHost, st));
  }
  CU(counted_sync(st));
  LVTRY(finish_pending(E));
  const uint32_t hc = E->h_counts[8];
  if (hc && (!hub_bound || hc > E->hub_count_cap)) {
    LVTRY(plan_hubs(hc));
    CU(cudaMemcpyAsync(E->h_counts, E->cls_count, 16 * sizeof(uint32_t),
                       cudaMemcpyDeviceToHost, st));
    CU(counted_sync(st));
  }
  g_trace.mark("  degree classes", (uint32_t)E->levels.size(), n);
  DispatchPlan& P = E->plan;
  memset(&P, 0, sizeof(P));
  P.cls_start[0] = 0;
  for (int c = 0; c < kClasses; c++) P.cls_start[c + 1] = P.cls_start[c] + E->h_counts[c];
  const uint32_t hs = P.cls_start[8];
  uint32_t hb = 0, hu = 0;
  uint64_t stage_total = 0, ct_total = 0;
  if (hc) {
    hb = E->h_counts[kHubTotals];
    hu = E->h_counts[kHubTotals + 1];
    memcpy(&stage_total, E->h_counts + kHubTotals + 2, sizeof(uint64_t));
    memcpy(&ct_total, E->h_counts + kHubTotals + 4, sizeof(uint64_t));
    if (hb == ~0u || hu == ~0u) return fail(LV_ERR_LIMIT, "hub plan: capacity exceeded");
  }
  P.hub_count = hc;
  P.hub_blocks = hb;
  H.units = hu;
  // dispatch units per class
  uint32_t u = 0;
  for (int c = 1; c <= 7; c++) {
    P.blk_start[c] = u;
    const uint32_t cnt = P.cls_start[c + 1] - P.cls_start[c];
    u += (cnt + class_per_unit(c) - 1) / class_per_unit(c);
  }
  P.blk_start[8] = u;
  u += P.hub_blocks;
  P.blk_start[9] = u;
  P.total_blocks = u;
  // partials: hub accumulators + 2 per dispatch block
  const size_t need_partials =
      hc + 2 * (size_t)std::max(dispatch_grid(P), pass_dispatch_grid()) + 16;
  if (need_partials > E->partials_cap) {
    E->partials_cap = 0;
    dfree(E->partials);
    CU(dalloc(&E->partials, need_partials));
    E->partials_cap = need_partials;
  }
  if (hc) {
    if (hb > E->hub_blocks_cap) {
      E->hub_blocks_cap = 0;
      dfree(E->hub_map);
      CU(dalloc(&E->hub_map, 2 * (size_t)hb));
      E->hub_blocks_cap = hb;
    }
    if (hu > E->hub_units_cap) {
      E->hub_units_cap = 0;
      dfree(H.blk_vertex);
      dfree(H.blk_chunk);
      dfree(H.blk_nchunks);
      dfree(H.unit_g);
      dfree(H.unit_c);
      CU(dalloc(&H.blk_vertex, hu));
      CU(dalloc(&H.blk_chunk, hu));
      CU(dalloc(&H.blk_nchunks, hu));
      CU(dalloc(&H.unit_g, hu));
      CU(dalloc(&H.unit_c, hu));
      E->hub_units_cap = hu;
    }
    // split/merge plan: staging copy of the hub rows, chunk table
    if (stage_total > E->hub_stage_cap) {
      E->hub_stage_cap = 0;
      dfree(H.stage);
      CU(dalloc(&H.stage, stage_total));
      E->hub_stage_cap = stage_total;
    }
    if (ct_total > E->hub_ct_cap) {
      E->hub_ct_cap = 0;
      dfree(H.ct);
      CU(dalloc(&H.ct, ct_total));
      E->hub_ct_cap = ct_total;
    }
    (count_launches(1), hub_fill_kernel<<<std::min<uint32_t>((hc + 7) / 8, 1184), 256, 0, st>>>(
        hc, hb, E->hub_chunk_start, H.unit_start, H.nparts, E->hub_map, H.blk_vertex,
        H.blk_chunk, H.blk_nchunks));
    CU(cudaGetLastError());
    CU(cudaMemsetAsync(H.best, 0, hc * sizeof(unsigned long long), st));
    CU(cudaMemsetAsync(H.own, 0, hc * sizeof(double), st));
    CU(cudaMemsetAsync(H.hot, 0, hc * sizeof(double), st));
    CU(cudaMemsetAsync(H.hot_any, 0, hc * sizeof(uint32_t), st));
    CU(cudaMemsetAsync(E->partials, 0, hc * sizeof(double), st));
  }
  if (E->batch) {
    // batched form: where each graph's run starts in every class list; the
    // hub list is never compacted
    CU(launch_class_graph_starts(E->order, P, E->goff_dev, E->n_graphs, E->cg, st));
    if (hc)
      CU(cudaMemcpyAsync(E->act_order + hs, E->order + hs, hc * sizeof(uint32_t),
                         cudaMemcpyDeviceToDevice, st));
  }
  g_trace.mark("  hub plan", (uint32_t)E->levels.size(), n);
  // entries per move class (byte counts of the kernel timings; profiling
  // only: the copy into the engine's pageable array blocks the host)
  if (E->profiling) {
    if (!E->d_class_deg) CU(dalloc(&E->d_class_deg, kClasses));
    CU(cudaMemsetAsync(E->d_class_deg, 0, kClasses * sizeof(unsigned long long), st));
    if (n) {
      (count_launches(1), class_degree_kernel<<<std::min<uint32_t>((n + 255) / 256, 1184), 256, 0, st>>>(
          E->off(), n, E->d_class_deg));
      CU(cudaGetLastError());
    }
    CU(cudaMemcpyAsync(E->class_deg, E->d_class_deg, kClasses * sizeof(uint64_t),
                       cudaMemcpyDeviceToHost, st));
  }
  // row sums, singleton state, m; then Q of the singleton partition.  A
  // single graph's level init also writes the row of every entry, for the
  // pass loop's modularity sweep (kept in the contraction's column scratch
  // until the level ends), and the incremental sweep's pass-start
  // communities (singletons)
  const LevelView L = E->view();
  const double Vd = (double)n, Ed = (double)E->e;
  cudaEvent_t t0 = prof_begin(E);
  CU(launch_level_init(L, E->order, P, hc ? E->hub_map : nullptr, E->partials,
                       E->batch ? nullptr : E->cb.tcol, E->batch ? nullptr : E->comm_start,
                       st));
  prof_end(E, t0, K_LEVEL_INIT, Ed * 4.0 + Vd * 32.0);
  t0 = prof_begin(E);
  CU(launch_modularity(L, E->order, P, hc ? E->hub_map : nullptr, E->partials, st));
  prof_end(E, t0, K_MODULARITY, Ed * 12.0 + Vd * 24.0);
  if (sync_scalars) {  // else the level graph's own synchronisation reads them
    CU(cudaMemcpyAsync(E->sc_host, E->sc, sizeof(LevelScalars),
                       cudaMemcpyDeviceToHost, st));
    CU(counted_sync(st));
    prof_collect(E);
  }
  g_trace.mark("  level init + Q0", (uint32_t)E->levels.size(), n);
  // tables of E->n vertices (blocking host copies above must be done
  // before the vectors go out of scope: synchronised)
  E->level_ready = true;
  return LV_OK;
}

lv_status issue_pass(lv_engine* E, const PassControl* ctl);

constexpr uint64_t kIncrementalMinEntries = 1ull << 23;

// The kernel of bucket b on this level: the tuned (or default) variant,
// except that a warp-per-vertex bucket with no more vertices than the block
// kernel has resident blocks gives each vertex a whole block -- there the
// launch lasts as long as one vertex's chain, which a block shortens
// (single graph; a union keeps its tuning).
uint8_t effective_variant(const lv_engine* E, int b) {
  const uint8_t v = E->tune[b];
  if (E->batch || b < 1 || b > 6) return v;
  if (v != KV_WARP128 && v != KV_WARP512) return v;
  const uint32_t cnt = E->plan.cls_start[b + 1] - E->plan.cls_start[b];
  return (cnt > 0 && cnt <= move_block_resident()) ? (uint8_t)KV_BLOCK : v;
}

// Writes the current level into the device pass descriptor (every pass
// kernel reads it at launch).
lv_status upload_desc(lv_engine* E, float min_gain) {
  PassDesc d{};
  d.L = E->view();
  const uint32_t* ord = E->batch ? E->act_order : E->order;
  d.A = dispatch_args(ord, E->plan, E->plan.hub_count ? E->hub_map : nullptr, E->partials);
  d.A.act_cnt = E->batch ? E->act_cnt : nullptr;
  d.prop = E->prop;
  d.full_order = E->order;
  d.H = E->hub;
  d.act_cnt = E->batch ? E->act_cnt : nullptr;
  d.act_order = E->act_order;
  d.cg = E->cg;
  d.cg_new = E->cg_new;
  d.n_graphs = E->batch ? E->n_graphs : 0u;
  // single graph: row ids built by prepare_level in the contraction's
  // column scratch, which is idle until the level's pass loop ends
  d.rowid = E->batch ? nullptr : E->cb.tcol;
  d.nnz = E->e;
  d.min_gain = (double)min_gain;
  d.max_passes = E->cfg.max_passes;
  for (int b = 0; b < 8; b++) d.tune[b] = effective_variant(E, b);
  d.loop = E->loop_state;
  d.fused = E->cfg.apply_launch ? 0u : 1u;
  // incremental sweeps only where a sweep is bound by DRAM: below 2^23
  // entries the level sits in L2 and the flat sweep over every entry costs
  // less than visiting the moved rows class by class (bench workload 5.68
  // -> 6.09 ms per run with it on every level; R-MAT 24 675 -> 652 ms)
  d.comm_start = (!E->batch && !E->cfg.modularity_full && E->e >= kIncrementalMinEntries)
                     ? E->comm_start
                     : nullptr;
  // through pinned memory: a copy from pageable memory would wait for the
  // stream first; the previous copy must have left the buffer
  CU(cudaEventSynchronize(E->desc_ev));
  *E->desc_host = d;
  CU(cudaMemcpyAsync(E->d_desc, E->desc_host, sizeof(d), cudaMemcpyHostToDevice, E->st));
  CU(cudaEventRecord(E->desc_ev, E->st));
  return LV_OK;
}

// Kernel class c (1..8) has vertices on this level.  A class empty at a
// single graph's level start stays empty through its passes, so its
// kernels are left out of the pass.  A union (batched and served forms)
// keeps every class: its class mix changes as graphs join and leave, and
// capturing and instantiating a level graph for each new mix cost more
// than the empty launches (served mix, 200 requests: 59.7 -> 64.0
// graphs/s, small-graph lane p50 546 -> 24 ms).
bool class_nonempty(const lv_engine* E, int c) {
  if (E->batch) return true;
  return c == 8 ? E->plan.hub_count > 0 : E->plan.cls_start[c + 1] > E->plan.cls_start[c];
}

// What a captured pass depends on besides the descriptor: the form
// (batched passes compact their lists), the rule, the tuning and which
// classes are non-empty.
uint64_t level_key(const lv_engine* E) {
  uint64_t k = (E->batch ? 1u : 0u) | ((uint64_t)(E->cfg.rule == LV_RULE_CUDA) << 1) |
               ((uint64_t)(E->cfg.gain == LV_GAIN_FP64) << 2) |
               ((uint64_t)(E->cfg.apply_launch != 0) << 3);
  for (int b = 1; b <= kBuckets; b++) k |= (uint64_t)effective_variant(E, b) << (4 * b);
  for (int c = 1; c <= 8; c++) k |= (uint64_t)class_nonempty(E, c) << (39 + c);
  return k;
}

constexpr size_t kLevelExecCache = 8;

void drop_level_exec(lv_engine* E) {
  for (const lv_engine::LevelExec& x : E->level_execs) cudaGraphExecDestroy(x.exec);
  E->level_execs.clear();
}

// Every pass of a level in one graph launch: [control init] -> WHILE
// { 7 Jacobi steps; modularity sweep + stop rule }.  The modularity
// kernel's last block evaluates the stop rule (modularity.cu:501-508) and
// sets the loop condition, so the host waits once per level instead of
// once per pass.  The kernels read the level from the descriptor, so the
// graph is captured once and replayed on every later level and run.
lv_status run_level_graph(lv_engine* E, float min_gain, bool wait = true) {
  LVTRY(upload_desc(E, min_gain));
  const uint64_t key = level_key(E);
  cudaGraphExec_t exec = nullptr;
  for (size_t i = 0; i < E->level_execs.size(); i++) {
    if (E->level_execs[i].key != key) continue;
    lv_engine::LevelExec hit = E->level_execs[i];  // most recently used goes last
    E->level_execs.erase(E->level_execs.begin() + (long)i);
    E->level_execs.push_back(hit);
    exec = hit.exec;
    E->level_launches = hit.launches;
    break;
  }
  if (!exec) {
    cudaGraph_t g = nullptr;
    CU(cudaGraphCreate(&g, 0));
    struct GraphGuard {
      cudaGraph_t g;
      ~GraphGuard() { if (g) cudaGraphDestroy(g); }
    } guard{g};
    t_capturing = true;
    t_tally = 0;
    // the loop's handle first: the init kernel sets its first condition
    cudaGraphConditionalHandle h;
    CU(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
    PassControl ictl{};
    ictl.use_handle = E->batch ? 0 : 1;
    ictl.handle = (unsigned long long)h;
    CU(cudaStreamBeginCaptureToGraph(E->st, g, nullptr, nullptr, 0,
                                     cudaStreamCaptureModeThreadLocal));
    cudaError_t ce = launch_pass_control_init(E->d_desc, &ictl, E->st);
    cudaGraph_t cap = nullptr;
    cudaError_t ce2 = cudaStreamEndCapture(E->st, &cap);
    t_capturing = false;
    CU(ce);
    CU(ce2);
    cudaGraphNode_t init_node = nullptr;
    size_t nn = 1;
    CU(cudaGraphGetNodes(g, &init_node, &nn));
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t cond_node = nullptr;
    CU(cudaGraphAddNode(&cond_node, g, &init_node, 1, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    PassControl ctl{};
    ctl.enabled = 1;
    ctl.use_handle = 1;
    ctl.handle = (unsigned long long)h;
    t_capturing = true;
    t_tally = 0;
    CU(cudaStreamBeginCaptureToGraph(E->st, body, nullptr, nullptr, 0,
                                     cudaStreamCaptureModeThreadLocal));
    E->capturing = true;
    lv_status s = issue_pass(E, &ctl);
    E->level_launches = t_tally;
    cudaGraph_t bcap = nullptr;
    ce = cudaStreamEndCapture(E->st, &bcap);
    t_capturing = false;
    E->capturing = false;
    E->pending.clear();
    if (s != LV_OK) return s;
    CU(ce);
    CU(cudaGraphInstantiate(&exec, g, 0));
    if (E->level_execs.size() >= kLevelExecCache) {
      cudaGraphExecDestroy(E->level_execs.front().exec);
      E->level_execs.erase(E->level_execs.begin());
    }
    E->level_execs.push_back({key, exec, E->level_launches});
    g_trace.mark("capture+instantiate", (uint32_t)E->levels.size(), E->n);
  }
  CU(cudaGraphLaunch(exec, E->st));
  CU(cudaMemcpyAsync(E->sc_host, E->sc, sizeof(LevelScalars), cudaMemcpyDeviceToHost,
                     E->st));
  if (!wait) return LV_OK;  // the caller's next synchronisation reads sc_host
  CU(counted_sync(E->st));
  g_trace.mark("graph run (all passes)", (uint32_t)E->levels.size(), E->n);
  return LV_OK;
}

// One pass (used when timing kernels: event nodes cannot live in a
// conditional body).  With graphs on, the first pass of a level is captured
// and every pass replays it.
lv_status run_pass(lv_engine* E, const PassControl* ctl = nullptr) {
  if (!E->cfg.use_graphs) return issue_pass(E, ctl);
  if (!E->pass_exec) {
    t_capturing = true;
    t_tally = 0;
    CU(cudaStreamBeginCapture(E->st, cudaStreamCaptureModeThreadLocal));
    E->capturing = true;
    lv_status s = issue_pass(E, ctl);
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(E->st, &g);
    E->capturing = false;
    t_capturing = false;
    if (s != LV_OK) {
      if (g) cudaGraphDestroy(g);
      return s;
    }
    CU(ce);
    ce = cudaGraphInstantiate(&E->pass_exec, g, 0);
    cudaGraphDestroy(g);
    CU(ce);
    E->pass_launches = t_tally;
    E->graph_timings.swap(E->pending);
    E->pending.clear();
  }
  CU(cudaGraphLaunch(E->pass_exec, E->st));
  count_launches((unsigned)E->pass_launches);
  return LV_OK;
}

int engine_mode(const lv_engine* E) {
  return move_mode(E->cfg.rule == LV_RULE_CUDA ? LV_RULE_CUDA_I : LV_RULE_PY_I,
                   E->cfg.gain == LV_GAIN_FP64 ? 1 : 0);
}

lv_status issue_pass(lv_engine* E, const PassControl* ctl) {
  const int rule = engine_mode(E);
  const PassDesc* D = E->d_desc;
  cudaStream_t st = E->st;
  // batched form: this pass visits only the graphs still moving
  if (E->batch) CU(launch_compact_active(D, st));
  // fused steps: step s reads copy s % 2 of the community state and leaves
  // every move up to its own in the other (StepIO); the first kernel of a
  // step re-applies the previous step's moves there
  const bool fused = !E->cfg.apply_launch;
  StepIO io{fused ? 1 : 0, 0, 0, 0, 1};  // pass_start: the first kernel of the pass
  int step = 0;
  // the kernels of classes empty on this level are left out (the level
  // graph is keyed by which classes are non-empty)
  for (int b = 1; b <= kBuckets; b++) {
    const bool hubs = b == 7 && class_nonempty(E, 8);
    if (!class_nonempty(E, b) && !hubs) continue;
    const uint32_t s = E->plan.cls_start[b];
    const uint32_t e = (b == 7) ? E->plan.cls_start[9] : E->plan.cls_start[b + 1];
    // algorithmic bytes: every entry's (col, w, comm[col]) and, per vertex,
    // order id, offset, comm, k, a_C(v) (FP64) and the proposal
    const double vb = (double)(e - s);
    const double v7 = (double)(E->plan.cls_start[b + 1] - s);
    cudaEvent_t t0;
    io.parity = fused ? (step & 1) : 0;
    if (class_nonempty(E, b)) {
      t0 = prof_begin(E);
      uint8_t kv[8];
      for (int i = 0; i < 8; i++) kv[i] = effective_variant(E, i);
      CU(launch_move_bucket(D, b, rule, kv, st, io));
      prof_end(E, t0, K_MOVE1 + b - 1, (double)E->class_deg[b] * 12.0 + v7 * 32.0);
      io.prev_lo = io.prev_hi = 0;  // re-applied by this launch
      io.pass_start = 0;
    }
    if (hubs) {
      t0 = prof_begin(E);
      CU(launch_move_bucket(D, 8, rule, nullptr, st, io));
      io.pass_start = 0;
      prof_end(E, t0, K_HUB,
               (double)E->class_deg[8] * 12.0 + (double)E->plan.hub_count * 32.0);
    }
    if (fused) {
      io.prev_lo = b;
      io.prev_hi = b == 7 ? 8 : b;
      step++;
    } else {
      t0 = prof_begin(E);
      CU(launch_apply_bucket(D, b, E->batch, st));
      prof_end(E, t0, K_APPLY, vb * 12.0);
    }
  }
  io.parity = fused ? (step & 1) : 0;
  cudaEvent_t t0 = prof_begin(E);
  CU(launch_modularity_pass(D, ctl, st, io));
  prof_end(E, t0, K_MODULARITY, (double)E->e * 12.0 + (double)E->n * 24.0);
  return LV_OK;
}

lv_status check_device_error(lv_engine* E) {
  if (E->sc_host->error == kErrBarrierTimeout) {
    return fail(LV_ERR_TIMEOUT, "a grid barrier wait of the level kernel gave up");
  }
  if (E->sc_host->error) {
    return fail(LV_ERR_LIMIT, "a device hash table overflowed (bounded probe gave up)");
  }
  return LV_OK;
}

// A single graph's level runs as one persistent kernel (the batched and
// served forms keep the per-kernel level graph: their passes compact the
// lists of graphs still moving).
bool use_level_kernel(const lv_engine* E) { return !E->batch && E->cfg.level_kernel; }

// Algorithmic bytes of one pass per timing group (as issue_pass counts them).
void pass_group_bytes(const lv_engine* E, double* out /*[K_COUNT]*/) {
  for (int i = 0; i < K_COUNT; i++) out[i] = 0.0;
  for (int b = 1; b <= kBuckets; b++) {
    const uint32_t s = E->plan.cls_start[b];
    const uint32_t e = (b == 7) ? E->plan.cls_start[9] : E->plan.cls_start[b + 1];
    const double v7 = (double)(E->plan.cls_start[b + 1] - s);
    out[K_MOVE1 + b - 1] = (double)E->class_deg[b] * 12.0 + v7 * 32.0;
    out[K_APPLY] += (double)(e - s) * 12.0;
  }
  out[K_HUB] = (double)E->class_deg[8] * 12.0 + (double)E->plan.hub_count * 32.0;
  out[K_MODULARITY] = (double)E->e * 12.0 + (double)E->n * 24.0;
}

// The level's pass loop in one cooperative launch of the persistent level
// kernel; the host waits once, for the level's result.
lv_status run_level_loop(lv_engine* E, float min_gain) {
  LVTRY(upload_desc(E, min_gain));
  memset(E->loop_host, 0, sizeof(LevelLoopState));
  E->loop_host->timing = E->profiling ? 1u : 0u;
  CU(cudaMemcpyAsync(E->loop_state, E->loop_host, sizeof(LevelLoopState),
                     cudaMemcpyHostToDevice, E->st));
  CU(launch_level_loop(E->d_desc, engine_mode(E), E->st));
  CU(cudaMemcpyAsync(E->sc_host, E->sc, sizeof(LevelScalars), cudaMemcpyDeviceToHost, E->st));
  if (E->profiling)
    CU(cudaMemcpyAsync(E->loop_host, E->loop_state, sizeof(LevelLoopState),
                       cudaMemcpyDeviceToHost, E->st));
  CU(counted_sync(E->st));
  if (E->profiling) {  // per-phase device time, as block 0 saw the barriers
    double bytes[K_COUNT];
    pass_group_bytes(E, bytes);
    const double passes = (double)E->sc_host->passes;
    for (int k = 0; k < kPhaseKinds; k++) {
      if (!E->loop_host->phase_cnt[k]) continue;
      E->kst[k].launches += E->loop_host->phase_cnt[k];
      E->kst[k].ms += (double)E->loop_host->phase_ns[k] * 1e-6;
      E->kst[k].bytes += bytes[k] * passes;
    }
  }
  g_trace.mark("level kernel (all passes)", (uint32_t)E->levels.size(), E->n);
  return LV_OK;
}

lv_status load_common(lv_engine* E, uint32_t n, uint64_t e) {
  drop_pass_graph(E);
  E->agg_pending = false;  // a new graph: nothing deferred is still wanted
  E->n0 = n;
  E->n = n;
  E->e = e;
  E->cur = -1;
  E->loaded = true;
  E->level_ready = false;
  E->finished = false;
  E->accepted = false;
  E->batch = false;
  E->n_graphs = 0;
  E->levels.clear();
  E->q_last = 0.0;
  CU(launch_fill_iota(E->assignment, n, E->st));  // setInitComm, utils.cu:67
  CU(cudaMemsetAsync(E->sc, 0, sizeof(LevelScalars), E->st));
  return LV_OK;
}

lv_status validate_sizes(uint32_t n, uint64_t e) {
  if (n >= 0xFFFFFFFFu) return fail(LV_ERR_LIMIT, "vertex count must be < 2^32-1");
  (void)e;
  return LV_OK;
}

// ---------------------------------------------------------------------------
// Batched form: many graphs as one block-diagonal union.  Every graph runs
// the reference's phase loop on its own (own m, modularity, stop rule);
// the kernels serve all graphs of a level at once.  A graph whose phase
// ends is finalised (its community ids made local) and dropped from the
// union at the next contraction.
// ---------------------------------------------------------------------------
lv_status batch_alloc(lv_engine* E, uint32_t G) {
  if (G <= E->graph_cap && E->gs) return LV_OK;
  E->graph_cap = 0;
  dfree(E->gs);
  dfree(E->goff_dev);
  dfree(E->gbase);
  dfree(E->gdrop);
  dfree(E->cg);
  dfree(E->cg_new);
  dfree(E->act_cnt);
  if (E->gs_host) cudaFreeHost(E->gs_host);
  E->gs_host = nullptr;
  CU(dalloc(&E->cg, (size_t)kMoveClasses * (G + 1)));
  CU(dalloc(&E->cg_new, (size_t)kMoveClasses * (G + 1)));
  CU(dalloc(&E->act_cnt, 16));
  CU(dalloc(&E->gs, G));
  CU(dalloc(&E->goff_dev, (size_t)G + 1));
  CU(dalloc(&E->gbase, G));
  CU(dalloc(&E->gdrop, G));
  CU(cudaMallocHost(&E->gs_host, sizeof(GraphState) * (G ? G : 1)));
  E->graph_cap = G;
  return LV_OK;
}

// One level's pass loop over every graph of the union; afterwards
// gs_host holds every graph's passes, stop flags and modularity values.
lv_status batch_passes(lv_engine* E, float min_gain) {
  if (!E->level_ready) LVTRY(prepare_level(E));
  if (E->cfg.use_graphs && !E->profiling) {
    LVTRY(run_level_graph(E, min_gain));
  } else {
    LVTRY(upload_desc(E, min_gain));
    CU(launch_pass_control_init(E->d_desc, nullptr, E->st));
    PassControl ctl{};
    ctl.enabled = 1;
    ctl.use_handle = 0;
    for (;;) {
      LVTRY(run_pass(E, &ctl));
      CU(cudaMemcpyAsync(E->sc_host, E->sc, sizeof(LevelScalars), cudaMemcpyDeviceToHost,
                         E->st));
      CU(counted_sync(E->st));
      if (E->pass_exec) prof_collect_graph(E);
      prof_collect(E);
      if (!E->sc_host->any_active) break;
    }
  }
  CU(cudaMemcpyAsync(E->gs_host, E->gs, sizeof(GraphState) * E->n_graphs,
                     cudaMemcpyDeviceToHost, E->st));
  CU(counted_sync(E->st));
  if (E->cfg.use_graphs && !E->profiling) {  // replays of the WHILE body
    uint32_t maxp = 0;
    for (uint32_t g = 0; g < E->n_graphs; g++) maxp = std::max(maxp, E->gs_host[g].passes);
    count_launches((unsigned)(1 + maxp * E->level_launches));
  }
  return check_device_error(E);
}

// A graph of the union: its input vertices carry `slot` in graph0 (and
// gbase[slot] finalises them), it owns `nv` consecutive vertices of the
// current level.
struct UnionGraph {
  uint32_t slot;
  uint32_t nv;
  uint32_t levels;  // move phases run so far
  uint8_t frozen;   // its run ended at the last contraction (merged nothing
                    // or reached max_levels); only its result is reported
  double q;         // modularity after its last move phase
};

// One level of the union.  Every graph that is not frozen runs its pass
// loop (modularity.cu:438-508, per graph); a graph whose run ends here --
// frozen, no edge weight, or a first pass below min gain -- has its input
// vertices' community ids written to `out` local to the graph (through the
// arena map graph0 -> gbase) and moves to `done`; the others are contracted
// (aggregation.cu:387-462) and stay in `graphs` with their new sizes, in
// union order.  The decisions are those run_loaded takes for one graph.
lv_status union_level(lv_engine* E, std::vector<UnionGraph>& graphs, float min_gain,
                      uint32_t* out, std::vector<UnionGraph>& done, uint64_t* processed) {
  cudaStream_t st = E->st;
  const uint32_t Gl = (uint32_t)graphs.size();
  E->n_graphs = Gl;
  std::vector<uint32_t> goff(Gl + 1, 0);
  bool all_frozen = true;
  for (uint32_t g = 0; g < Gl; g++) {
    goff[g + 1] = goff[g] + graphs[g].nv;
    all_frozen = all_frozen && graphs[g].frozen;
  }
  if (goff[Gl] != E->n) return fail(LV_ERR_STATE, "union sizes out of step");
  if (!all_frozen) {
    std::vector<GraphState> init(Gl);
    memset(init.data(), 0, sizeof(GraphState) * Gl);
    for (uint32_t g = 0; g < Gl; g++) init[g].frozen = graphs[g].frozen;
    CU(cudaMemcpyAsync(E->gs, init.data(), sizeof(GraphState) * Gl, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(E->goff_dev, goff.data(), (Gl + 1) * sizeof(uint32_t),
                       cudaMemcpyHostToDevice, st));
    CU(launch_graph_ids(E->goff_dev, Gl, E->n, E->gid, st));
    g_trace.mark("union: level start", (uint32_t)E->levels.size(), E->n);
    LVTRY(batch_passes(E, min_gain));  // synchronises: init/goff may go
    g_trace.mark("union: passes", (uint32_t)E->levels.size(), E->n);
  }
  std::vector<uint32_t> base(E->graph_cap, 0xFFFFFFFFu), drop(Gl, 0u);
  std::vector<uint8_t> last(Gl, 0);
  bool any_continue = false;
  uint64_t lvl_passes = 0;
  for (uint32_t g = 0; g < Gl; g++) {
    UnionGraph& u = graphs[g];
    bool ended = true;
    if (!u.frozen) {
      const GraphState& s = E->gs_host[g];
      u.levels++;
      lvl_passes = std::max<uint64_t>(lvl_passes, s.passes);
      if (s.passes == 0) u.q = 0.0;                 // no edge weight: nothing moves
      else if (s.first_fail) u.q = s.q_before;      // the pass's moves are discarded
      else {
        u.q = s.q;
        ended = false;
        last[g] = E->cfg.max_levels && u.levels >= E->cfg.max_levels;
      }
    }
    if (ended) {
      base[u.slot] = goff[g];
      drop[g] = 1u;
    }
    any_continue = any_continue || !ended;
  }
  if (!all_frozen) {
    lv_level_info info{};
    info.n_vertices = E->n;
    info.n_entries = E->e;
    info.passes = (uint32_t)lvl_passes;
    info.moved = any_continue ? 1u : 0u;
    E->levels.push_back(info);
    if (processed) *processed += lvl_passes * E->e;
  }
  // finalise the graphs that end here
  CU(cudaMemcpyAsync(E->gbase, base.data(), E->graph_cap * sizeof(uint32_t),
                     cudaMemcpyHostToDevice, st));
  CU(launch_finalize_graphs(E->assignment, E->n0, E->graph0, E->gbase, out, st));
  std::vector<UnionGraph> kept;
  for (uint32_t g = 0; g < Gl; g++) (drop[g] ? done : kept).push_back(graphs[g]);
  if (!any_continue) {
    CU(counted_sync(st));
    graphs.clear();
    E->n = 0;
    E->e = 0;
    E->level_ready = false;
    return LV_OK;
  }
  // contract the graphs that go on; the others leave the union
  CU(cudaMemcpyAsync(E->gdrop, drop.data(), Gl * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  CU(launch_drop_graphs(E->comm_sz, E->gid, E->n, E->gdrop, st));
  E->accepted = true;
  g_trace.mark("union: finalize", (uint32_t)E->levels.size(), E->n);
  LVTRY(lv_phase_aggregate(E));  // synchronises
  g_trace.mark("union: contract", (uint32_t)E->levels.size(), E->n);
  // new offsets: the new id of each kept graph's first vertex (flag_id is
  // the exclusive scan of non-empty communities in old-id order)
  std::vector<uint32_t> first;
  for (uint32_t g = 0; g < Gl; g++)
    if (!drop[g]) first.push_back(goff[g]);
  const uint32_t Gn = (uint32_t)first.size();
  CU(cudaMemcpyAsync(E->gbase, first.data(), Gn * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  CU(launch_gather_u32(E->cb.flag_id, E->gbase, Gn, E->goff_dev, st));
  std::vector<uint32_t> ng(Gn + 1);
  CU(cudaMemcpyAsync(ng.data(), E->goff_dev, Gn * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  CU(counted_sync(st));
  ng[Gn] = E->n;
  for (uint32_t g = 0, i = 0; g < Gl; g++) {
    if (drop[g]) continue;
    UnionGraph& u = kept[i];
    const uint32_t nv = ng[i + 1] - ng[i];
    // a level that merged nothing would repeat forever (min gain <= 0)
    u.frozen = (nv == u.nv || last[g]) ? 1u : 0u;
    u.nv = nv;
    i++;
  }
  graphs.swap(kept);
  return LV_OK;
}

}  // namespace

// Drives the batched run; see lv_batch_run_device in the C ABI.
static lv_status batch_run(lv_engine* E, uint32_t G, const uint64_t* goff_in,
                           float min_gain, uint32_t* d_out, double* q_out,
                           uint32_t* levels_out, lv_result* res) {
  LVTRY(batch_alloc(E, G));
  cudaStream_t st = E->st;
  const uint32_t n0 = E->n0;
  if (n0 > E->act_order_cap) {
    E->act_order_cap = 0;
    dfree(E->act_order);
    CU(dalloc(&E->act_order, n0));
    E->act_order_cap = n0;
  }
  // input vertex -> graph (its slot)
  std::vector<uint32_t> goff(G + 1);
  for (uint32_t g = 0; g <= G; g++) goff[g] = (uint32_t)goff_in[g];
  CU(cudaMemcpyAsync(E->goff_dev, goff.data(), (G + 1) * sizeof(uint32_t),
                     cudaMemcpyHostToDevice, st));
  CU(launch_graph_ids(E->goff_dev, G, n0, E->graph0, st));
  std::vector<UnionGraph> graphs(G), done;
  for (uint32_t g = 0; g < G; g++) graphs[g] = UnionGraph{g, goff[g + 1] - goff[g], 0u, 0u, 0.0};
  E->batch = true;
  cudaEvent_t a0, a1;
  CU(cudaEventCreate(&a0));
  CU(cudaEventCreate(&a1));
  CU(cudaEventRecord(a0, st));
  uint64_t processed = 0;
  lv_status status = LV_OK;
  while (!graphs.empty() && status == LV_OK)
    status = union_level(E, graphs, min_gain, d_out, done, &processed);
  CU(cudaEventRecord(a1, st));
  CU(cudaEventSynchronize(a1));
  float alg = 0.0f;
  cudaEventElapsedTime(&alg, a0, a1);
  cudaEventDestroy(a0);
  cudaEventDestroy(a1);
  E->batch = false;
  E->finished = true;
  if (status != LV_OK) return status;
  uint64_t n_comm = 0;
  for (const UnionGraph& u : done) {
    if (q_out) q_out[u.slot] = u.q;
    if (levels_out) levels_out[u.slot] = u.levels;
    n_comm += u.nv;
  }
  if (res) {
    res->modularity = 0.0;
    res->n_vertices = n0;
    res->n_communities = (uint32_t)n_comm;
    res->n_levels = (uint32_t)E->levels.size();
    res->edges_processed = processed;
    res->alg_ms = alg;
    res->copy_ms = 0.0f;
  }
  return LV_OK;
}

// ---------------------------------------------------------------------------
// Served form: continuous batching.  Requests queue on submit, routed by
// size to one of up to four lanes; a lane is one union of resident graphs
// on its own engine and stream.  Every step of a lane admits its queued
// graphs that fit its share of the device budget (FIFO), appends them to
// its union at the level boundary -- so a new graph's level 0 runs beside
// the resident graphs' later levels -- and runs one union level; graphs
// whose run ends are finalised, copied out and leave at once, freeing their
// slots and memory.  Lanes keep small graphs from being paced by large
// ones (a union level lasts as long as its slowest graph's pass loop) and,
// stepped by worker threads, run concurrently on the device.  A graph's
// kernels read only its own rows and state, so its result equals a run of
// it alone.
// ---------------------------------------------------------------------------
namespace {

// Device bytes that a resident vertex / adjacency entry may hold across the
// engine's buffers (CSR ping-pong, per-vertex state, contraction and hub
// staging, scans), for admission against the budget.
constexpr uint64_t kServeBytesPerVertex = 192;
constexpr uint64_t kServeBytesPerEntry = 40;

struct ServeRequest {
  uint64_t ticket = 0;
  const lv_graph* g = nullptr;  // the caller's graph, alive until polled
  uint32_t n = 0;               // its sizes
  uint64_t nnz = 0;
  double t_submit = 0.0, t_admit = -1.0, t_done = -1.0;
  uint32_t lane = 0, slot = 0, a0 = 0;  // lane, slot and arena range while resident
  double q = 0.0;
  uint32_t levels = 0, n_comm = 0;
  std::vector<uint32_t> assignment;
};

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// One union of resident graphs on its own engine (and stream).
struct ServeLane {
  lv_engine* E = nullptr;
  bool solo = false;         // one request at a time, single-graph path
  uint64_t max_entries = 0;  // routing: requests with at most this many entries
  uint32_t cap_n = 0, slot_cap = 0;
  uint64_t cap_e = 0;
  std::deque<ServeRequest*> queue;  // guarded by lv_server::mu
  std::vector<ServeRequest*> by_slot;
  std::vector<uint32_t> free_slots;
  std::vector<UnionGraph> graphs;   // resident, in union order (lane thread only)
  uint32_t arena_used = 0;          // input-vertex arena bump pointer
  uint64_t res_n = 0, res_e = 0;    // input sizes of the resident graphs (under mu)
  uint32_t n_res = 0;               // resident graphs (under mu)
  uint32_t* out = nullptr;          // arena-indexed local ids
  uint64_t steps = 0, admitted = 0, completed = 0;
  std::thread worker;
  cudaStream_t stream = nullptr;  // created for the lane (priority by size)
};

}  // namespace

struct lv_server {
  lv_serve_config cfg{};
  std::vector<ServeLane*> lanes;
  std::mutex mu;  // queues, finished, counters shared with submit / poll
  std::condition_variable cv_work, cv_done;
  std::deque<ServeRequest*> finished;
  uint64_t next_ticket = 1;
  uint32_t busy = 0;  // lanes in the middle of a step
  bool stop = false;
  lv_status bg_status = LV_OK;  // first failure of a lane worker
  std::string bg_error;
  std::chrono::steady_clock::time_point t0;
};

namespace {

// Moves the resident graphs' arena ranges to the front (the arena is a bump
// allocator; finished graphs leave holes).
lv_status serve_compact(ServeLane* L) {
  lv_engine* E = L->E;
  cudaStream_t st = E->st;
  std::vector<ServeRequest*> live;
  for (const UnionGraph& u : L->graphs) live.push_back(L->by_slot[u.slot]);
  std::sort(live.begin(), live.end(),
            [](const ServeRequest* a, const ServeRequest* b) { return a->a0 < b->a0; });
  uint32_t w = 0;
  uint32_t* tmp = E->cb.cursor;  // contraction scratch, idle between levels
  for (ServeRequest* r : live) {
    CU(cudaMemcpyAsync(tmp + w, E->assignment + r->a0, (size_t)r->n * sizeof(uint32_t),
                       cudaMemcpyDeviceToDevice, st));
    r->a0 = w;
    w += r->n;
  }
  if (w) {
    CU(cudaMemcpyAsync(E->assignment, tmp, (size_t)w * sizeof(uint32_t),
                       cudaMemcpyDeviceToDevice, st));
  }
  for (ServeRequest* r : live) CU(launch_fill_u32(E->graph0 + r->a0, r->n, r->slot, st));
  L->arena_used = w;
  E->n0 = w;
  return LV_OK;
}

// Appends request r's graph to the lane's union (rows after the current
// level's last vertex) and gives it an arena range and a slot.
lv_status serve_append(ServeLane* L, ServeRequest* r) {
  lv_engine* E = L->E;
  cudaStream_t st = E->st;
  const lv_graph& g = *r->g;
  if (L->arena_used + g.n > L->cap_n) LVTRY(serve_compact(L));
  if (E->cur < 0) {  // first graph: the union lives in the contraction buffers
    E->cur = 0;
    E->n = 0;
    E->e = 0;
  }
  const int c = E->cur;
  const uint32_t vb = E->n;
  const uint64_t eb = E->e;
  CU(cudaMemcpyAsync(E->c_off[c] + vb, g.off.data(), ((size_t)g.n + 1) * sizeof(uint64_t),
                     cudaMemcpyHostToDevice, st));
  CU(launch_add_u64(E->c_off[c] + vb, (size_t)g.n + 1, eb, st));
  if (g.nnz) {
    CU(cudaMemcpyAsync(E->c_col[c] + eb, g.col.data(), g.nnz * sizeof(uint32_t),
                       cudaMemcpyHostToDevice, st));
    CU(launch_add_u32(E->c_col[c] + eb, g.nnz, vb, st));
    CU(cudaMemcpyAsync(E->c_w[c] + eb, g.w.data(), g.nnz * sizeof(float),
                       cudaMemcpyHostToDevice, st));
  }
  r->slot = L->free_slots.back();
  L->free_slots.pop_back();
  L->by_slot[r->slot] = r;
  r->a0 = L->arena_used;
  CU(launch_iota_from(E->assignment + r->a0, g.n, vb, st));
  CU(launch_fill_u32(E->graph0 + r->a0, g.n, r->slot, st));
  L->arena_used += g.n;
  E->n0 = L->arena_used;
  E->n += g.n;
  E->e += g.nnz;
  E->level_ready = false;
  L->graphs.push_back(UnionGraph{r->slot, g.n, 0u, 0u, 0.0});
  return LV_OK;
}

// A solo lane's step: its oldest queued request, run alone through the
// single-graph path (lv_run: upload, every level, assignment).
lv_status solo_step(lv_server* S, ServeLane* L) {
  lv_engine* E = L->E;
  ServeRequest* r = nullptr;
  {
    std::lock_guard<std::mutex> lock(S->mu);
    if (L->queue.empty()) return LV_OK;
    r = L->queue.front();
    L->queue.pop_front();
    L->res_n += r->n;
    L->res_e += r->nnz;
    L->n_res++;
  }
  r->t_admit = ms_since(S->t0);
  L->admitted++;
  lv_result res{};
  LVTRY(lv_run(E, r->g, S->cfg.min_gain, &res));
  r->assignment.resize(r->n);
  LVTRY(lv_get_assignment(E, r->assignment.data(), r->n));
  r->q = res.modularity;
  r->levels = res.n_levels;
  r->n_comm = res.n_communities;
  E->levels.clear();
  L->steps++;
  {
    std::lock_guard<std::mutex> lock(S->mu);
    r->t_done = ms_since(S->t0);
    L->res_n -= r->n;
    L->res_e -= r->nnz;
    L->n_res--;
    L->completed++;
    S->finished.push_back(r);
  }
  S->cv_done.notify_all();
  return LV_OK;
}

// One step of a lane: admissions, then one level of its union.
lv_status lane_step(lv_server* S, ServeLane* L) {
  if (L->solo) return solo_step(S, L);
  lv_engine* E = L->E;
  cudaSetDevice(E->device);
  AllocScope alloc_scope(E);
  std::vector<ServeRequest*> adm;
  {
    std::lock_guard<std::mutex> lock(S->mu);
    uint64_t tn = L->res_n, te = L->res_e;
    size_t slots = L->free_slots.size();
    while (!L->queue.empty()) {
      ServeRequest* r = L->queue.front();
      if (!slots || tn + r->n > L->cap_n || te + r->nnz > L->cap_e) break;
      adm.push_back(r);
      L->queue.pop_front();
      tn += r->n;
      te += r->nnz;
      slots--;
    }
    L->res_n = tn;  // reserved now, released when the graph leaves
    L->res_e = te;
    L->n_res += (uint32_t)adm.size();
  }
  g_trace.reset();
  for (ServeRequest* r : adm) {
    LVTRY(serve_append(L, r));
    r->t_admit = ms_since(S->t0);
    L->admitted++;
  }
  g_trace.mark("serve: admit + append", (uint32_t)adm.size(), E->n);
  if (L->graphs.empty()) return LV_OK;
  std::vector<UnionGraph> done;
  LVTRY(union_level(E, L->graphs, S->cfg.min_gain, L->out, done, nullptr));
  E->levels.clear();
  L->steps++;
  for (const UnionGraph& u : done) {
    ServeRequest* r = L->by_slot[u.slot];
    r->assignment.resize(r->n);
    CU(cudaMemcpyAsync(r->assignment.data(), L->out + r->a0, (size_t)r->n * sizeof(uint32_t),
                       cudaMemcpyDeviceToHost, E->st));
    r->q = u.q;
    r->levels = u.levels;
    r->n_comm = u.nv;
  }
  CU(counted_sync(E->st));
  const double now = ms_since(S->t0);
  {
    std::lock_guard<std::mutex> lock(S->mu);
    for (const UnionGraph& u : done) {
      ServeRequest* r = L->by_slot[u.slot];
      r->t_done = now;
      L->by_slot[u.slot] = nullptr;
      L->free_slots.push_back(u.slot);
      L->res_n -= r->n;
      L->res_e -= r->nnz;
      L->n_res--;
      L->completed++;
      S->finished.push_back(r);
    }
  }
  if (!done.empty()) S->cv_done.notify_all();
  if (L->graphs.empty()) {  // every arena range is free
    L->arena_used = 0;
    E->n0 = 0;
  }
  return LV_OK;
}

// Background mode: a lane steps while it has queued or resident graphs.
void lane_worker(lv_server* S, ServeLane* L) {
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_work.wait(lk, [&] { return S->stop || !L->queue.empty() || !L->graphs.empty(); });
      if (S->stop) return;
      S->busy++;
    }
    const lv_status st = lane_step(S, L);
    std::lock_guard<std::mutex> lock(S->mu);
    S->busy--;
    if (st != LV_OK) {
      if (S->bg_status == LV_OK) {
        S->bg_status = st;
        S->bg_error = lv_last_error();
      }
      S->cv_done.notify_all();
      return;  // the lane stops; the server reports the error from now on
    }
    S->cv_done.notify_all();
  }
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* lv_status_string(lv_status s) {
  switch (s) {
    case LV_OK: return "ok";
    case LV_ERR_ARG: return "invalid argument";
    case LV_ERR_IO: return "Error opening file";
    case LV_ERR_PARSE: return "malformed Matrix Market input";
    case LV_ERR_NOMEM: return "out of memory";
    case LV_ERR_CUDA: return "CUDA error";
    case LV_ERR_STATE: return "call out of order";
    case LV_ERR_LIMIT: return "size limit exceeded";
    case LV_ERR_TIMEOUT: return "device wait timed out";
  }
  return "unknown status";
}

const char* lv_last_error(void) { return g_last_error.c_str(); }

int lv_abi_version(void) { return LV_ABI_VERSION; }

void lv_config_default(lv_config* cfg) {
  if (!cfg) return;
  memset(cfg, 0, sizeof(*cfg));
  cfg->device = 0;
  cfg->rule = LV_RULE_PY;
  cfg->max_passes = 0;
  cfg->max_levels = 0;
  cfg->use_graphs = 1;
  cfg->stream = nullptr;
  cfg->gain = LV_GAIN_FP32;
  cfg->level_kernel = 0;
  cfg->contract_sort = 0;
  cfg->apply_launch = 0;
  cfg->modularity_full = 0;
}

lv_status lv_engine_create(const lv_config* cfg, lv_engine** out) {
  if (!out) return fail(LV_ERR_ARG, "out is NULL");
  *out = nullptr;
  lv_engine* E = new (std::nothrow) lv_engine();
  if (!E) return fail(LV_ERR_NOMEM, "engine allocation failed");
  if (cfg) {
    E->cfg = *cfg;
  } else {
    lv_config_default(&E->cfg);
  }
  if (E->cfg.rule != LV_RULE_PY && E->cfg.rule != LV_RULE_CUDA) {
    delete E;
    return fail(LV_ERR_ARG, "unknown rule");
  }
  if (E->cfg.gain != LV_GAIN_FP32 && E->cfg.gain != LV_GAIN_FP64) {
    delete E;
    return fail(LV_ERR_ARG, "unknown gain arithmetic");
  }
  if (E->cfg.max_passes == 0) E->cfg.max_passes = 100000;
  E->device = E->cfg.device;
  cudaError_t ce = cudaSetDevice(E->device);
  if (ce != cudaSuccess) {
    delete E;
    return cuda_fail(ce, "cudaSetDevice");
  }
  ce = configure_kernels();
  if (ce != cudaSuccess) {
    delete E;
    return cuda_fail(ce, "configure_kernels");
  }
  {  // the engine's own pool; freed blocks stay in it for the next growth
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = E->device;
    ce = cudaMemPoolCreate(&E->pool, &props);
    if (ce != cudaSuccess) {
      delete E;
      return cuda_fail(ce, "cudaMemPoolCreate");
    }
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(E->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  if (E->cfg.stream) {
    E->st = (cudaStream_t)E->cfg.stream;
  } else {
    ce = cudaStreamCreateWithFlags(&E->st, cudaStreamNonBlocking);
    if (ce != cudaSuccess) {
      cudaMemPoolDestroy(E->pool);
      delete E;
      return cuda_fail(ce, "cudaStreamCreate");
    }
    E->own_stream = true;
  }
  if ((ce = cudaMalloc(&E->sc, sizeof(LevelScalars))) != cudaSuccess ||
      (ce = cudaMalloc(&E->d_desc, sizeof(PassDesc))) != cudaSuccess ||
      (ce = cudaMalloc(&E->loop_state, sizeof(LevelLoopState))) != cudaSuccess ||
      (ce = cudaMallocHost(&E->loop_host, sizeof(LevelLoopState))) != cudaSuccess ||
      (ce = cudaMallocHost(&E->sc_host, sizeof(LevelScalars))) != cudaSuccess ||
      (ce = cudaMallocHost(&E->h_counts, 32 * sizeof(uint32_t))) != cudaSuccess ||
      (ce = cudaEventCreate(&E->ev0)) != cudaSuccess ||
      (ce = cudaEventCreate(&E->ev1)) != cudaSuccess ||
      (ce = cudaEventCreate(&E->agg_ev0)) != cudaSuccess ||
      (ce = cudaEventCreateWithFlags(&E->desc_ev, cudaEventDisableTiming)) != cudaSuccess ||
      (ce = cudaMallocHost(&E->desc_host, sizeof(PassDesc))) != cudaSuccess ||
      (ce = cudaEventCreate(&E->agg_ev1)) != cudaSuccess ||
      (ce = cudaMallocHost(&E->h_pending, 2 * sizeof(uint64_t))) != cudaSuccess) {
    lv_engine_destroy(E);
    return cuda_fail(ce, "engine set-up");
  }
  memset(E->sc_host, 0, sizeof(LevelScalars));
  *out = E;
  return LV_OK;
}

void lv_engine_destroy(lv_engine* E) {
  if (!E) return;
  AllocScope alloc_scope(E);
  cudaSetDevice(E->device);
  if (E->st) counted_sync(E->st);
  drop_pass_graph(E);
  drop_level_exec(E);
  free_state(E);
  dfree(E->gs);
  dfree(E->goff_dev);
  dfree(E->gbase);
  dfree(E->gdrop);
  dfree(E->batch_out);
  dfree(E->act_order);
  dfree(E->cg);
  dfree(E->cg_new);
  dfree(E->act_cnt);
  if (E->gs_host) cudaFreeHost(E->gs_host);
  prof_collect(E);
  for (cudaEvent_t ev : E->ev_free) cudaEventDestroy(ev);
  E->ev_free.clear();
  dfree(E->d_class_deg);
  if (E->sc) cudaFree(E->sc);
  if (E->d_desc) cudaFree(E->d_desc);
  if (E->loop_state) cudaFree(E->loop_state);
  if (E->agg_ev0) cudaEventDestroy(E->agg_ev0);
  if (E->desc_ev) cudaEventDestroy(E->desc_ev);
  if (E->desc_host) cudaFreeHost(E->desc_host);
  if (E->agg_ev1) cudaEventDestroy(E->agg_ev1);
  if (E->h_pending) cudaFreeHost(E->h_pending);
  if (E->loop_host) cudaFreeHost(E->loop_host);
  if (E->sc_host) cudaFreeHost(E->sc_host);
  if (E->h_counts) cudaFreeHost(E->h_counts);
  if (E->ev0) cudaEventDestroy(E->ev0);
  if (E->ev1) cudaEventDestroy(E->ev1);
  if (E->st) counted_sync(E->st);  // the frees above are stream-ordered
  if (E->pool) cudaMemPoolDestroy(E->pool);
  if (E->own_stream && E->st) cudaStreamDestroy(E->st);
  delete E;
}

lv_status lv_engine_load(lv_engine* E, const lv_graph* g) {
  AllocScope alloc_scope(E);
  if (!E || !g) return fail(LV_ERR_ARG, "NULL engine or graph");
  LVTRY(validate_sizes(g->n, g->nnz));
  cudaSetDevice(E->device);
  LVTRY(ensure_capacity(E, g->n, g->nnz, true));
  E->in_off = E->own_off;
  E->in_col = E->own_col;
  E->in_w = E->own_w;
  CU(cudaMemcpyAsync(E->own_off, g->off.data(), ((size_t)g->n + 1) * sizeof(uint64_t),
                     cudaMemcpyHostToDevice, E->st));
  if (g->nnz) {
    CU(cudaMemcpyAsync(E->own_col, g->col.data(), g->nnz * sizeof(uint32_t),
                       cudaMemcpyHostToDevice, E->st));
    CU(cudaMemcpyAsync(E->own_w, g->w.data(), g->nnz * sizeof(float),
                       cudaMemcpyHostToDevice, E->st));
  }
  return load_common(E, g->n, g->nnz);
}

// Host edge lines -> device -> the reference reader's CSR built on the
// device (sort by row) in the engine's input buffers.
static lv_status load_edges_common(lv_engine* E, uint32_t n, uint64_t m, const uint32_t* src,
                                   const uint32_t* dst, const float* w) {
  if (n >= 0xFFFFFFFFu) return fail(LV_ERR_LIMIT, "vertex count must be < 2^32-1");
  if (m >= (1ull << 31)) return fail(LV_ERR_LIMIT, "at most 2^31 - 1 edge lines");
  cudaSetDevice(E->device);
  LVTRY(ensure_capacity(E, n, 2 * m, true));
  uint32_t *d_src = nullptr, *d_dst = nullptr;
  float* d_w = nullptr;
  struct Tmp {
    uint32_t*& a;
    uint32_t*& b;
    float*& c;
    ~Tmp() {
      dfree(a);
      dfree(b);
      dfree(c);
    }
  } tmp{d_src, d_dst, d_w};
  CU(dalloc(&d_src, m));
  CU(dalloc(&d_dst, m));
  if (w) CU(dalloc(&d_w, m));
  if (m) {
    CU(cudaMemcpyAsync(d_src, src, m * sizeof(uint32_t), cudaMemcpyHostToDevice, E->st));
    CU(cudaMemcpyAsync(d_dst, dst, m * sizeof(uint32_t), cudaMemcpyHostToDevice, E->st));
    if (w) CU(cudaMemcpyAsync(d_w, w, m * sizeof(float), cudaMemcpyHostToDevice, E->st));
  }
  uint64_t nnz = 0;
  uint32_t bad = 0;
  CU(csr_from_edges_device(n, m, d_src, d_dst, d_w, E->own_off, E->own_col, E->own_w, &nnz, &bad,
                           E->st));
  if (bad) return fail(LV_ERR_PARSE, "vertex index exceeds the vertex count");
  E->in_off = E->own_off;
  E->in_col = E->own_col;
  E->in_w = E->own_w;
  return load_common(E, n, nnz);
}

lv_status lv_engine_load_edges(lv_engine* E, uint32_t n, uint64_t m, const uint32_t* src,
                               const uint32_t* dst, const float* w) {
  AllocScope alloc_scope(E);
  if (!E || (m && (!src || !dst))) return fail(LV_ERR_ARG, "NULL argument");
  return load_edges_common(E, n, m, src, dst, w);
}

lv_status lv_engine_load_mtx(lv_engine* E, const char* path) {
  AllocScope alloc_scope(E);
  if (!E || !path) return fail(LV_ERR_ARG, "NULL argument");
  uint32_t n = 0;
  std::vector<uint32_t> src, dst;
  std::vector<float> ws;
  LVTRY(lvb_parse_mtx(path, &n, src, dst, ws));
  return load_edges_common(E, n, src.size(), src.data(), dst.data(), ws.data());
}

lv_status lv_csr_from_edges_device(uint32_t n, uint64_t m, const uint32_t* d_src,
                                   const uint32_t* d_dst, const float* d_w, uint64_t* d_off,
                                   uint32_t* d_col, float* d_w_out, uint64_t* nnz,
                                   void* stream) {
  if (!d_off || !nnz || (m && (!d_src || !d_dst || !d_col || !d_w_out)))
    return fail(LV_ERR_ARG, "NULL argument");
  if (n >= 0xFFFFFFFFu) return fail(LV_ERR_LIMIT, "vertex count must be < 2^32-1");
  if (m >= (1ull << 31)) return fail(LV_ERR_LIMIT, "at most 2^31 - 1 edge lines");
  uint32_t bad = 0;
  uint64_t h_nnz = 0;
  CU(csr_from_edges_device(n, m, d_src, d_dst, d_w, d_off, d_col, d_w_out, &h_nnz, &bad,
                           static_cast<cudaStream_t>(stream)));
  if (bad) return fail(LV_ERR_PARSE, "vertex index exceeds the vertex count");
  *nnz = h_nnz;
  return LV_OK;
}

lv_status lv_engine_load_device(lv_engine* E, uint32_t n, uint64_t nnz,
                                const uint64_t* d_off, const uint32_t* d_col,
                                const float* d_w) {
  AllocScope alloc_scope(E);
  if (!E || !d_off || (nnz && (!d_col || !d_w)))
    return fail(LV_ERR_ARG, "NULL engine or device buffer");
  LVTRY(validate_sizes(n, nnz));
  cudaSetDevice(E->device);
  LVTRY(ensure_capacity(E, n, nnz, false));
  E->in_off = const_cast<uint64_t*>(d_off);
  E->in_col = const_cast<uint32_t*>(d_col);
  E->in_w = const_cast<float*>(d_w);
  return load_common(E, n, nnz);
}

// A level's move phase.  With `speculate` (the whole-run loop of a single
// graph), the contraction's front is launched behind the level graph
// before its result is known, and one synchronisation reads both: the
// level's scalars and the contraction's class sizes.  A level that moved
// nothing drops the front (it wrote only contraction scratch).
static lv_status phase_move(lv_engine* E, float min_gain, int* more, double* q,
                            bool speculate) {
  AllocScope alloc_scope(E);
  if (!E) return fail(LV_ERR_ARG, "NULL engine");
  if (!E->loaded) return fail(LV_ERR_STATE, "no graph loaded");
  if (E->finished) return fail(LV_ERR_STATE, "the run has ended; load a graph again");
  cudaSetDevice(E->device);
  E->front_ready = false;
  CU(cudaEventRecord(E->ev0, E->st));
  g_trace.reset();
  // the level graph reads the level's m and initial Q on the device and the
  // host after the whole level: no synchronisation between set-up and loop
  const bool graph_path = E->cfg.use_graphs && !E->profiling && !use_level_kernel(E);
  if (!E->level_ready) LVTRY(prepare_level(E, !graph_path));
  g_trace.mark("prepare", (uint32_t)E->levels.size(), E->n);
  cudaEvent_t ev_prep = take_event(E);
  CU(cudaEventRecord(ev_prep, E->st));
  lv_level_info info{};
  info.n_vertices = E->n;
  info.n_entries = E->e;
  const bool spec = speculate && graph_path && !E->batch && !E->cfg.contract_sort;
  if (graph_path) LVTRY(run_level_graph(E, min_gain, !spec));  // reads sc_host
  if (spec) {
    CU(cudaEventRecord(E->ev1, E->st));  // the level's end
    CU(cudaEventRecord(E->agg_ev0, E->st));
    CU(contract_front(E->view(), E->e, E->cb, E->scan, E->st, grow_tables, E));
    CU(counted_sync(E->st));
    E->front_ready = true;
  }
  const double m64 = E->sc_host->m64;
  double act = graph_path ? E->sc_host->q_start : E->sc_host->q, old = act;
  info.q_start = act;
  int ret = 1;
  uint32_t passes = 0;
  if (!(m64 > 0.0)) {
    // no edge weight: nothing can move (the reference loops forever here)
    ret = 0;
    act = old = 0.0;
    info.q_start = 0.0;
  } else if (use_level_kernel(E)) {
    LVTRY(run_level_loop(E, min_gain));
    LVTRY(check_device_error(E));
    passes = E->sc_host->passes;
    ret = E->sc_host->first_fail ? 0 : 1;
    act = E->sc_host->q;
    old = E->sc_host->q_before;
  } else if (graph_path) {
    LVTRY(check_device_error(E));
    passes = E->sc_host->passes;
    ret = E->sc_host->first_fail ? 0 : 1;
    act = E->sc_host->q;
    old = E->sc_host->q_before;
    count_launches((unsigned)(1 + passes * E->level_launches));
  } else {
    LVTRY(upload_desc(E, min_gain));
    bool first = true;
    do {
      LVTRY(run_pass(E));
      CU(cudaMemcpyAsync(E->sc_host, E->sc, sizeof(LevelScalars),
                         cudaMemcpyDeviceToHost, E->st));
      CU(counted_sync(E->st));
      if (E->pass_exec) prof_collect_graph(E);
      prof_collect(E);
      LVTRY(check_device_error(E));
      old = act;
      act = E->sc_host->q;
      passes++;
      if (first && act - old < (double)min_gain) ret = 0;  // modularity.cu:503
      first = false;
    } while (act - old >= (double)min_gain && passes < E->cfg.max_passes);
  }
  E->accepted = ret != 0;  // modularity.cu:515-517 (applied at aggregation)
  if (!ret) E->front_ready = false;
  if (!spec) CU(cudaEventRecord(E->ev1, E->st));
  CU(cudaEventSynchronize(E->ev1));
  float ms = 0.0f, prep_ms = 0.0f;
  cudaEventElapsedTime(&ms, E->ev0, E->ev1);
  cudaEventElapsedTime(&prep_ms, E->ev0, ev_prep);
  E->ev_free.push_back(ev_prep);
  info.passes = passes;
  info.moved = (uint32_t)ret;
  info.q_end = act;
  info.move_ms = ms;
  info.prepare_ms = prep_ms;
  E->levels.push_back(info);
  if (!ret) E->finished = true;
  E->q_last = ret ? act : old;
  if (more) *more = ret;
  if (q) *q = E->q_last;
  return LV_OK;
}

lv_status lv_phase_move(lv_engine* E, float min_gain, int* more, double* q) {
  return phase_move(E, min_gain, more, q, false);
}

// Entry-sized buffers of the contraction by sorting, grown on demand.
lv_status ensure_sort_buffers(lv_engine* E, uint64_t nnz) {
  SortBuffers& S = E->sb;
  if (nnz <= S.cap && S.keys[0]) return LV_OK;
  S.cap = 0;  // zeroed before the frees (see grow_tables)
  dfree(S.keys[0]);
  dfree(S.keys[1]);
  dfree(S.vals[0]);
  dfree(S.vals[1]);
  dfree(S.pos);
  dfree(S.counts);
  dfree(E->sb_scan);
  S.scan.buf = nullptr;
  const size_t cap = std::max<uint64_t>(nnz, 1024);
  CU(dalloc(&S.keys[0], cap));
  CU(dalloc(&S.keys[1], cap));
  CU(dalloc(&S.vals[0], cap));
  CU(dalloc(&S.vals[1], cap));
  CU(dalloc(&S.pos, cap));
  CU(dalloc(&S.counts, radix_sort_scratch_words(cap)));
  S.scan.bytes = scan_scratch_bytes(cap + 1024);
  CU(dalloc(&E->sb_scan, S.scan.bytes));
  S.scan.buf = E->sb_scan;
  S.cap = cap;
  return LV_OK;
}

lv_status lv_phase_aggregate(lv_engine* E) {
  AllocScope alloc_scope(E);
  if (!E) return fail(LV_ERR_ARG, "NULL engine");
  if (!E->loaded || !E->level_ready) return fail(LV_ERR_STATE, "no move phase to aggregate");
  cudaSetDevice(E->device);
  // a single graph outside profiling defers the reads that follow the
  // contraction to the next level's first synchronisation
  const bool defer = !E->batch && !E->profiling && !E->cfg.contract_sort;
  const bool front = E->front_ready;  // launched and read with the level's result
  E->front_ready = false;
  if (!front) CU(cudaEventRecord(defer ? E->agg_ev0 : E->ev0, E->st));
  const int next = (E->cur == 0) ? 1 : 0;
  ContractResult r{};
  cudaEvent_t t0 = prof_begin(E);
  g_trace.reset();
  if (!E->batch && E->cfg.contract_sort) {
    LVTRY(ensure_sort_buffers(E, E->e));
    CU(contract_level_sort(E->view(), E->e, E->cb, E->sb, E->scan, E->c_off[next],
                           E->c_col[next], E->c_w[next], &r, E->st));
  } else if (front) {
    CU(contract_back(E->view(), E->e, E->cb, E->scan, E->c_off[next], E->c_col[next],
                     E->c_w[next], &r, E->st, grow_tables, E, defer));
  } else {
    CU(contract_level(E->view(), E->e, E->cb, E->scan, E->c_off[next], E->c_col[next],
                      E->c_w[next], &r, E->st, grow_tables, E, defer));
  }
  g_trace.mark("contract", (uint32_t)E->levels.size(), E->n);
  // B_agg = E*12 + V*(off + comm + new id + member) + E'*8 + (V'+1)*off
  prof_end(E, t0, K_CONTRACT,
           (double)E->e * 12.0 + (double)E->n * 20.0 + (double)r.new_nnz * 8.0 +
               ((double)r.new_n + 1.0) * 8.0);
  // graphVertToComm then graphVertToNewComm (modularity.cu:51-56,
  // aggregation.cu:380-385) in one gather: cnew[v] = new_id[comm[v]]
  CU(launch_compose(E->assignment, E->n0, E->cb.cnew, E->st));
  E->accepted = false;
  if (defer) {
    CU(cudaEventRecord(E->agg_ev1, E->st));
    drop_pass_graph(E);
    E->cur = next;
    E->n = r.new_n;
    E->agg_pending = true;  // E->e, the error flag and the time come at the next sync
    E->level_ready = false;
    return LV_OK;
  }
  CU(cudaEventRecord(E->ev1, E->st));
  CU(cudaEventSynchronize(E->ev1));
  CU(cudaMemcpyAsync(E->sc_host, E->sc, sizeof(LevelScalars), cudaMemcpyDeviceToHost, E->st));
  CU(counted_sync(E->st));
  LVTRY(check_device_error(E));
  prof_collect(E);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, E->ev0, E->ev1);
  if (!E->levels.empty()) E->levels.back().aggregate_ms = ms;
  drop_pass_graph(E);
  E->cur = next;
  E->n = r.new_n;
  E->e = r.new_nnz;
  E->level_ready = false;
  return LV_OK;
}

static lv_status run_loaded(lv_engine* E, float min_gain, lv_result* res) {
  // a contraction front launched by this loop is consumed by it: never
  // left for a later entry point, whatever path the loop leaves by
  struct FrontGuard {
    lv_engine* E;
    ~FrontGuard() { E->front_ready = false; }
  } front_guard{E};
  CU(cudaEventRecord(E->ev0, E->st));
  cudaEvent_t a0, a1;
  CU(cudaEventCreate(&a0));
  CU(cudaEventCreate(&a1));
  CU(cudaEventRecord(a0, E->st));
  double q = 0.0;
  uint64_t processed = 0;
  for (;;) {
    int more = 0;
    lv_status s = phase_move(E, min_gain, &more, &q, true);
    if (s != LV_OK) {
      cudaEventDestroy(a0);
      cudaEventDestroy(a1);
      return s;
    }
    processed += (uint64_t)E->levels.back().passes * E->levels.back().n_entries;
    if (!more) break;
    const uint32_t before = E->n;
    s = lv_phase_aggregate(E);
    if (s != LV_OK) {
      cudaEventDestroy(a0);
      cudaEventDestroy(a1);
      return s;
    }
    if (E->n == before) {  // merged nothing (threshold <= 0): stop
      E->finished = true;
      break;
    }
    if (E->cfg.max_levels && E->levels.size() >= E->cfg.max_levels) {
      E->finished = true;
      break;
    }
  }
  {
    const lv_status ps = resolve_pending(E);  // a last contraction's reads
    if (ps != LV_OK) {
      cudaEventDestroy(a0);
      cudaEventDestroy(a1);
      return ps;
    }
  }
  CU(cudaEventRecord(a1, E->st));
  CU(cudaEventSynchronize(a1));
  float alg = 0.0f;
  cudaEventElapsedTime(&alg, a0, a1);
  cudaEventDestroy(a0);
  cudaEventDestroy(a1);
  if (res) {
    res->modularity = q;
    res->n_vertices = E->n0;
    res->n_communities = E->n;
    res->n_levels = (uint32_t)E->levels.size();
    res->edges_processed = processed;
    res->alg_ms = alg;
  }
  return LV_OK;
}

lv_status lv_run(lv_engine* E, const lv_graph* g, float min_gain, lv_result* res) {
  AllocScope alloc_scope(E);
  if (!E || !g) return fail(LV_ERR_ARG, "NULL engine or graph");
  cudaSetDevice(E->device);
  cudaEvent_t c0, c1;
  CU(cudaEventCreate(&c0));
  CU(cudaEventCreate(&c1));
  CU(cudaEventRecord(c0, E->st));
  lv_status s = lv_engine_load(E, g);
  if (s != LV_OK) {
    cudaEventDestroy(c0);
    cudaEventDestroy(c1);
    return s;
  }
  CU(cudaEventRecord(c1, E->st));  // the run starts behind the copies, no host wait
  s = run_loaded(E, min_gain, res);  // returns after the stream has finished
  float copy = 0.0f;
  if (s == LV_OK && cudaEventSynchronize(c1) == cudaSuccess)
    cudaEventElapsedTime(&copy, c0, c1);
  cudaEventDestroy(c0);
  cudaEventDestroy(c1);
  if (s == LV_OK && res) res->copy_ms = copy;
  return s;
}

lv_status lv_run_device(lv_engine* E, uint32_t n, uint64_t nnz, const uint64_t* d_off,
                        const uint32_t* d_col, const float* d_w, float min_gain,
                        uint32_t* d_assignment, lv_result* res) {
  AllocScope alloc_scope(E);
  if (!E) return fail(LV_ERR_ARG, "NULL engine");
  LVTRY(lv_engine_load_device(E, n, nnz, d_off, d_col, d_w));
  LVTRY(run_loaded(E, min_gain, res));
  if (res) res->copy_ms = 0.0f;
  if (d_assignment && n) {
    if (E->accepted) {
      CU(launch_gather(d_assignment, E->assignment, n, E->comm, E->st));
    } else {
      CU(cudaMemcpyAsync(d_assignment, E->assignment, (size_t)n * sizeof(uint32_t),
                         cudaMemcpyDeviceToDevice, E->st));
    }
    CU(counted_sync(E->st));
  }
  return LV_OK;
}

lv_status lv_get_assignment(lv_engine* E, uint32_t* out, size_t n) {
  if (E) LVTRY(resolve_pending(E));
  AllocScope alloc_scope(E);
  if (!E || (!out && n)) return fail(LV_ERR_ARG, "NULL argument");
  if (!E->loaded) return fail(LV_ERR_STATE, "no graph loaded");
  if (n != E->n0) return fail(LV_ERR_ARG, "buffer length must equal the input vertex count");
  cudaSetDevice(E->device);
  if (n) {
    const uint32_t* src = E->assignment;
    if (E->accepted) {  // the level's moves count: read comm[assignment]
      CU(launch_gather(E->cb.members, E->assignment, n, E->comm, E->st));
      src = E->cb.members;
    }
    CU(cudaMemcpyAsync(out, src, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, E->st));
    CU(counted_sync(E->st));
  }
  return LV_OK;
}

lv_status lv_get_communities(lv_engine* E, uint32_t* out, size_t cap, uint32_t* n_comm) {
  if (E) LVTRY(resolve_pending(E));
  AllocScope alloc_scope(E);
  if (!E || !n_comm) return fail(LV_ERR_ARG, "NULL argument");
  if (!E->loaded) return fail(LV_ERR_STATE, "no graph loaded");
  cudaSetDevice(E->device);
  const uint32_t n = E->n0;
  // the final communities are dense ids < the level's vertex count
  const uint32_t c = n ? E->n : 0u;
  *n_comm = c;
  const size_t need = (size_t)c + 1 + n;
  if (!out) return LV_OK;  // size query
  if (cap < need) return fail(LV_ERR_ARG, "buffer shorter than n_communities + 1 + n");
  uint32_t* part = E->assignment;
  if (E->accepted && n) {  // the level's moves count: comm[assignment]
    CU(launch_gather(E->cb.members, E->assignment, n, E->comm, E->st));
    part = E->cb.members;
  }
  uint32_t* d_out = nullptr;
  CU(dalloc(&d_out, need));
  cudaError_t ce = group_by_community(part, n, c, d_out, E->st);
  if (ce == cudaSuccess)
    ce = cudaMemcpyAsync(out, d_out, need * sizeof(uint32_t), cudaMemcpyDeviceToHost, E->st);
  if (ce == cudaSuccess) ce = counted_sync(E->st);
  dfree(d_out);
  CU(ce);
  return LV_OK;
}

lv_status lv_get_levels(lv_engine* E, lv_level_info* out, uint32_t cap, uint32_t* count) {
  if (E) LVTRY(resolve_pending(E));
  if (!E) return fail(LV_ERR_ARG, "NULL engine");
  const uint32_t nl = (uint32_t)E->levels.size();
  if (count) *count = nl;
  if (out)
    for (uint32_t i = 0; i < nl && i < cap; i++) out[i] = E->levels[i];
  return LV_OK;
}

lv_status lv_get_level_size(lv_engine* E, uint32_t* n, uint64_t* e) {
  if (E) LVTRY(resolve_pending(E));
  if (!E) return fail(LV_ERR_ARG, "NULL engine");
  if (n) *n = E->n;
  if (e) *e = E->e;
  return LV_OK;
}

lv_status lv_get_level_state(lv_engine* E, uint32_t* comm, uint32_t* comm_size,
                             float* weighted_degree) {
  if (E) LVTRY(resolve_pending(E));
  AllocScope alloc_scope(E);
  if (!E) return fail(LV_ERR_ARG, "NULL engine");
  if (!E->loaded) return fail(LV_ERR_STATE, "no graph loaded");
  cudaSetDevice(E->device);
  if (!E->level_ready) LVTRY(prepare_level(E));
  const size_t n = E->n;
  if (n) {
    if (comm) CU(cudaMemcpyAsync(comm, E->comm, n * 4, cudaMemcpyDeviceToHost, E->st));
    if (comm_size)
      CU(cudaMemcpyAsync(comm_size, E->comm_sz, n * 4, cudaMemcpyDeviceToHost, E->st));
    if (weighted_degree)
      CU(cudaMemcpyAsync(weighted_degree, E->k, n * 4, cudaMemcpyDeviceToHost, E->st));
  }
  CU(counted_sync(E->st));
  return LV_OK;
}

lv_status lv_get_level_csr(lv_engine* E, uint64_t* offsets, uint32_t* cols,
                           float* weights) {
  if (E) LVTRY(resolve_pending(E));
  AllocScope alloc_scope(E);
  if (!E) return fail(LV_ERR_ARG, "NULL engine");
  if (!E->loaded) return fail(LV_ERR_STATE, "no graph loaded");
  cudaSetDevice(E->device);
  if (offsets)
    CU(cudaMemcpyAsync(offsets, E->off(), ((size_t)E->n + 1) * 8, cudaMemcpyDeviceToHost,
                       E->st));
  if (E->e) {
    if (cols) CU(cudaMemcpyAsync(cols, E->col(), E->e * 4, cudaMemcpyDeviceToHost, E->st));
    if (weights)
      CU(cudaMemcpyAsync(weights, E->wts(), E->e * 4, cudaMemcpyDeviceToHost, E->st));
  }
  CU(counted_sync(E->st));
  return LV_OK;
}

lv_status lv_set_level_comm(lv_engine* E, const uint32_t* comm) {
  if (E) LVTRY(resolve_pending(E));
  AllocScope alloc_scope(E);
  if (!E || !comm) return fail(LV_ERR_ARG, "NULL argument");
  if (!E->loaded) return fail(LV_ERR_STATE, "no graph loaded");
  cudaSetDevice(E->device);
  for (uint32_t i = 0; i < E->n; i++)
    if (comm[i] >= E->n) return fail(LV_ERR_ARG, "community id out of range");
  if (!E->level_ready) LVTRY(prepare_level(E));
  if (E->n) CU(cudaMemcpyAsync(E->comm, comm, (size_t)E->n * 4, cudaMemcpyHostToDevice, E->st));
  CU(launch_recount(E->view(), E->st));
  if (E->n) {  // the second copy of the state starts equal to the first
    const size_t n = E->n;
    CU(cudaMemcpyAsync(E->comm_alt, E->comm, n * 4, cudaMemcpyDeviceToDevice, E->st));
    CU(cudaMemcpyAsync(E->sz_alt, E->comm_sz, n * 4, cudaMemcpyDeviceToDevice, E->st));
    CU(cudaMemcpyAsync(E->tot_alt, E->tot, n * 8, cudaMemcpyDeviceToDevice, E->st));
    CU(cudaMemcpyAsync(E->comm_start, E->comm, n * 4, cudaMemcpyDeviceToDevice, E->st));
  }
  CU(launch_modularity(E->view(), E->order, E->plan,
                       E->plan.hub_count ? E->hub_map : nullptr, E->partials, E->st));
  CU(cudaMemcpyAsync(E->sc_host, E->sc, sizeof(LevelScalars), cudaMemcpyDeviceToHost,
                     E->st));
  CU(counted_sync(E->st));
  E->accepted = true;
  return LV_OK;
}

lv_status lv_modularity_fp64(lv_engine* E, const uint32_t* partition, double* q) {
  if (E) LVTRY(resolve_pending(E));
  AllocScope alloc_scope(E);
  if (!E || !partition || !q) return fail(LV_ERR_ARG, "NULL argument");
  if (!E->loaded) return fail(LV_ERR_STATE, "no graph loaded");
  cudaSetDevice(E->device);
  for (uint32_t i = 0; i < E->n; i++)
    if (partition[i] >= E->n) return fail(LV_ERR_ARG, "community id out of range");
  uint32_t* d_part = E->cb.cursor;
  double* d_tot = reinterpret_cast<double*>(E->cb.comm_deg);
  double* d_out = reinterpret_cast<double*>(E->cb.new_deg);
  if (E->n) CU(cudaMemcpyAsync(d_part, partition, (size_t)E->n * 4, cudaMemcpyHostToDevice, E->st));
  CU(launch_modularity_of(E->view(), d_part, d_tot, d_out, E->st));
  double h[3] = {0, 0, 0};
  CU(cudaMemcpyAsync(h, d_out, sizeof(h), cudaMemcpyDeviceToHost, E->st));
  CU(counted_sync(E->st));
  const double m = h[2] / 2.0;
  *q = (m > 0.0) ? h[0] / (2.0 * m) - h[1] / (4.0 * m * m) : 0.0;
  return LV_OK;
}

lv_status lv_set_profiling(lv_engine* E, int on) {
  if (E) LVTRY(resolve_pending(E));
  if (!E) return fail(LV_ERR_ARG, "NULL engine");
  E->profiling = on != 0;
  return LV_OK;
}

lv_status lv_get_kernel_stats(lv_engine* E, lv_kernel_stat* out, uint32_t cap,
                              uint32_t* count) {
  if (!E) return fail(LV_ERR_ARG, "NULL engine");
  if (count) *count = K_COUNT;
  if (out) {
    for (uint32_t i = 0; i < K_COUNT && i < cap; i++) {
      memset(&out[i], 0, sizeof(out[i]));
      strncpy(out[i].name, kKName[i], sizeof(out[i].name) - 1);
      out[i].launches = E->kst[i].launches;
      out[i].total_ms = E->kst[i].ms;
      out[i].bytes = E->kst[i].bytes;
    }
  }
  return LV_OK;
}

lv_status lv_batch_run_device(lv_engine* E, uint32_t n_graphs, const uint64_t* graph_offsets,
                              uint32_t n_vertices, uint64_t n_entries, const uint64_t* d_offsets,
                              const uint32_t* d_cols, const float* d_weights, float min_gain,
                              uint32_t* d_assignment, double* modularity, uint32_t* levels,
                              lv_result* res) {
  AllocScope alloc_scope(E);
  if (!E || !graph_offsets || !d_assignment || (n_graphs && !modularity))
    return fail(LV_ERR_ARG, "NULL argument");
  if (n_graphs == 0) return fail(LV_ERR_ARG, "no graphs");
  if (graph_offsets[0] != 0 || graph_offsets[n_graphs] != n_vertices)
    return fail(LV_ERR_ARG, "graph offsets must run from 0 to the vertex count");
  for (uint32_t g = 0; g < n_graphs; g++)
    if (graph_offsets[g + 1] < graph_offsets[g])
      return fail(LV_ERR_ARG, "graph offsets must be non-decreasing");
  LVTRY(lv_engine_load_device(E, n_vertices, n_entries, d_offsets, d_cols, d_weights));
  return batch_run(E, n_graphs, graph_offsets, min_gain, d_assignment, modularity, levels, res);
}

lv_status lv_batch_run(lv_engine* E, uint32_t n_graphs, const lv_graph* const* graphs,
                       float min_gain, uint32_t* assignment, double* modularity,
                       uint32_t* levels, lv_result* res) {
  AllocScope alloc_scope(E);
  if (!E || !graphs || !assignment || !modularity) return fail(LV_ERR_ARG, "NULL argument");
  if (n_graphs == 0) return fail(LV_ERR_ARG, "no graphs");
  // pack the graphs into one block-diagonal CSR (vertex ids offset per graph)
  std::vector<uint64_t> goff(n_graphs + 1, 0), eoff(n_graphs + 1, 0);
  for (uint32_t g = 0; g < n_graphs; g++) {
    if (!graphs[g]) return fail(LV_ERR_ARG, "NULL graph");
    goff[g + 1] = goff[g] + graphs[g]->n;
    eoff[g + 1] = eoff[g] + graphs[g]->nnz;
  }
  if (goff[n_graphs] >= 0xFFFFFFFFull) return fail(LV_ERR_LIMIT, "too many vertices in the batch");
  const uint32_t N = (uint32_t)goff[n_graphs];
  const uint64_t NNZ = eoff[n_graphs];
  cudaSetDevice(E->device);
  LVTRY(ensure_capacity(E, N, NNZ, true));
  E->in_off = E->own_off;
  E->in_col = E->own_col;
  E->in_w = E->own_w;
  // the union is assembled on the device: every graph's rows are copied
  // into place and shifted by its vertex / entry offsets (a graph's last
  // offset and the next graph's first are the same value)
  cudaStream_t st = E->st;
  for (uint32_t g = 0; g < n_graphs; g++) {
    const lv_graph* h = graphs[g];
    const uint32_t vb = (uint32_t)goff[g];
    const uint64_t eb = eoff[g];
    CU(cudaMemcpyAsync(E->own_off + vb, h->off.data(), ((size_t)h->n + 1) * sizeof(uint64_t),
                       cudaMemcpyHostToDevice, st));
    CU(launch_add_u64(E->own_off + vb, (size_t)h->n + 1, eb, st));
    if (h->nnz) {
      CU(cudaMemcpyAsync(E->own_col + eb, h->col.data(), h->nnz * sizeof(uint32_t),
                         cudaMemcpyHostToDevice, st));
      CU(launch_add_u32(E->own_col + eb, h->nnz, vb, st));
      CU(cudaMemcpyAsync(E->own_w + eb, h->w.data(), h->nnz * sizeof(float),
                         cudaMemcpyHostToDevice, st));
    }
  }
  LVTRY(load_common(E, N, NNZ));
  if (N > E->batch_out_cap) {
    E->batch_out_cap = 0;
    dfree(E->batch_out);
    CU(dalloc(&E->batch_out, N));
    E->batch_out_cap = N;
  }
  uint32_t* d_out = E->batch_out;
  LVTRY(batch_run(E, n_graphs, goff.data(), min_gain, d_out, modularity, levels, res));
  CU(cudaMemcpyAsync(assignment, d_out, (size_t)N * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                     E->st));
  CU(counted_sync(E->st));
  return LV_OK;
}

// ---- served form ----------------------------------------------------------
void lv_serve_config_default(lv_serve_config* c) {
  if (!c) return;
  memset(c, 0, sizeof(*c));
  c->min_gain = 1e-6f;
  c->budget_bytes = 8ull << 30;
  c->max_graphs = 0;
  c->n_lanes = 4;
  c->lane_max_entries[0] = 1ull << 18;
  c->lane_max_entries[1] = 1ull << 22;
  c->lane_max_entries[2] = ~0ull;
  c->lane_max_entries[3] = ~0ull;
  c->lane_share[0] = 0.10f;
  c->lane_share[1] = 0.30f;
  c->lane_share[2] = 0.30f;
  c->lane_share[3] = 0.30f;
  c->background = 1;
  c->lane_solo = 0xCu;  // lanes 2 and 3
}

lv_status lv_serve_create(const lv_config* cfg, const lv_serve_config* scfg, lv_server** out) {
  if (!out || !scfg) return fail(LV_ERR_ARG, "NULL argument");
  *out = nullptr;
  if (scfg->n_lanes < 1 || scfg->n_lanes > 4) return fail(LV_ERR_ARG, "n_lanes must be 1..4");
  double share_sum = 0.0;
  for (uint32_t i = 0; i < scfg->n_lanes; i++) {
    if (!(scfg->lane_share[i] > 0.0f)) return fail(LV_ERR_ARG, "every lane needs a budget share");
    if (i && scfg->lane_max_entries[i] < scfg->lane_max_entries[i - 1])
      return fail(LV_ERR_ARG, "lane_max_entries must ascend");
    share_sum += scfg->lane_share[i];
  }
  const uint64_t per_v = kServeBytesPerVertex, per_e = kServeBytesPerEntry;
  lv_server* S = new (std::nothrow) lv_server();
  if (!S) return fail(LV_ERR_NOMEM, "server allocation failed");
  S->cfg = *scfg;
  S->cfg.lane_max_entries[scfg->n_lanes - 1] = ~0ull;  // the last lane takes the rest
  for (uint32_t i = scfg->n_lanes - 1; i > 0; i--)  // so do lanes with the same bound
    if (scfg->lane_max_entries[i - 1] == scfg->lane_max_entries[scfg->n_lanes - 1])
      S->cfg.lane_max_entries[i - 1] = ~0ull;
  for (uint32_t i = 0; i < scfg->n_lanes; i++) {
    const uint64_t budget = (uint64_t)((double)scfg->budget_bytes * scfg->lane_share[i] / share_sum);
    if (budget < 64 * (per_v + per_e)) {
      lv_serve_destroy(S);
      return fail(LV_ERR_ARG, "budget too small");
    }
    ServeLane* L = new (std::nothrow) ServeLane();
    if (!L) {
      lv_serve_destroy(S);
      return fail(LV_ERR_NOMEM, "lane allocation failed");
    }
    S->lanes.push_back(L);
    L->max_entries = S->cfg.lane_max_entries[i];
    // lanes of smaller graphs get higher stream priority, so their short
    // kernels are scheduled ahead of a large lane's blocks as SMs free up
    lv_config lc;
    if (cfg) lc = *cfg; else lv_config_default(&lc);
    if (!lc.stream) {
      int least = 0, greatest = 0;
      cudaSetDevice(lc.device);
      cudaDeviceGetStreamPriorityRange(&least, &greatest);
      const int span = least - greatest;  // greatest is the numerically lower
      const int prio = scfg->n_lanes > 1
                           ? greatest + (int)((int64_t)span * i / (scfg->n_lanes - 1))
                           : least;
      cudaError_t ce = cudaStreamCreateWithPriority(&L->stream, cudaStreamNonBlocking, prio);
      if (ce != cudaSuccess) {
        lv_serve_destroy(S);
        return cuda_fail(ce, "cudaStreamCreateWithPriority");
      }
      lc.stream = L->stream;
    }
    lv_status st = lv_engine_create(&lc, &L->E);
    if (st != LV_OK) {
      lv_serve_destroy(S);
      return st;
    }
    lv_engine* E = L->E;
    // a fifth of the lane's budget for per-vertex state, the rest for adjacency
    uint64_t cap_n = std::min<uint64_t>(budget / 5 / per_v, 0xFFFFFFF0ull);
    L->cap_n = (uint32_t)cap_n;
    L->cap_e = (budget - cap_n * per_v) / per_e;
    L->slot_cap = scfg->max_graphs ? scfg->max_graphs : 4096;
    L->solo = (scfg->lane_solo >> i) & 1u;
    if (L->solo) {  // no union: the engine allocates per request
      L->slot_cap = 1;
      L->by_slot.assign(1, nullptr);
      continue;
    }
    auto setup = [&]() -> lv_status {
      AllocScope alloc_scope(E);
      LVTRY(ensure_capacity(E, L->cap_n, L->cap_e, false));
      LVTRY(batch_alloc(E, L->slot_cap));
      CU(dalloc(&E->act_order, L->cap_n));
      E->act_order_cap = L->cap_n;
      CU(dalloc(&L->out, L->cap_n));
      // every id a stale arena entry can hold stays a valid index: compose
      // (cnew[assignment]) runs over the whole arena, holes included
      CU(cudaMemsetAsync(E->cb.cnew, 0, (size_t)L->cap_n * sizeof(uint32_t), E->st));
      CU(cudaMemsetAsync(E->sc, 0, sizeof(LevelScalars), E->st));
      CU(counted_sync(E->st));
      return LV_OK;
    };
    st = setup();
    if (st != LV_OK) {
      lv_serve_destroy(S);
      return st;
    }
    E->loaded = true;
    E->batch = true;
    E->cur = -1;
    E->n = 0;
    E->e = 0;
    E->n0 = 0;
    L->by_slot.assign(L->slot_cap, nullptr);
    for (uint32_t k = L->slot_cap; k > 0; k--) L->free_slots.push_back(k - 1);
  }
  S->t0 = std::chrono::steady_clock::now();
  if (scfg->background) {
    try {
      for (ServeLane* L : S->lanes) L->worker = std::thread(lane_worker, S, L);
    } catch (const std::system_error&) {
      lv_serve_destroy(S);
      return fail(LV_ERR_NOMEM, "worker thread start failed");
    }
  }
  *out = S;
  return LV_OK;
}

lv_status lv_serve_submit(lv_server* S, const lv_graph* g, uint64_t* ticket) {
  if (!S || !g) return fail(LV_ERR_ARG, "NULL server or graph");
  // the first size bound that holds the graph; among the lanes sharing that
  // bound (a group), the one with the fewest entries resident or queued
  uint32_t lane = ~0u;
  {
    std::lock_guard<std::mutex> lock(S->mu);
    uint64_t bound = 0, best_load = ~0ull;
    for (uint32_t i = 0; i < S->lanes.size(); i++) {
      const ServeLane* L = S->lanes[i];
      if (g->nnz > L->max_entries || g->n > L->cap_n || g->nnz > L->cap_e) continue;
      if (lane != ~0u && L->max_entries != bound) break;
      uint64_t load = L->res_e;
      for (const ServeRequest* q : L->queue) load += q->nnz;
      if (lane == ~0u || load < best_load) {
        lane = i;
        bound = L->max_entries;
        best_load = load;
      }
    }
  }
  if (lane == ~0u) return fail(LV_ERR_LIMIT, "graph exceeds the server's device budget");
  ServeRequest* r = new (std::nothrow) ServeRequest();
  if (!r) return fail(LV_ERR_NOMEM, "request allocation failed");
  r->g = g;  // not copied: the caller keeps it alive until the result is polled
  r->n = g->n;
  r->nnz = g->nnz;
  r->lane = lane;
  {
    std::lock_guard<std::mutex> lock(S->mu);
    r->ticket = S->next_ticket++;
    r->t_submit = ms_since(S->t0);
    if (g->n == 0) {  // nothing to run
      r->t_admit = r->t_done = r->t_submit;
      S->finished.push_back(r);
    } else {
      S->lanes[lane]->queue.push_back(r);
    }
    if (ticket) *ticket = r->ticket;
  }
  S->cv_work.notify_all();
  S->cv_done.notify_all();
  return LV_OK;
}

namespace {
void serve_counts(lv_server* S, uint32_t* resident, uint32_t* queued) {
  uint32_t r = 0, q = 0;
  for (const ServeLane* L : S->lanes) {
    r += L->n_res;
    q += (uint32_t)L->queue.size();
  }
  if (resident) *resident = r;
  if (queued) *queued = q;
}
}  // namespace

lv_status lv_serve_step(lv_server* S, uint32_t* resident, uint32_t* queued) {
  if (!S) return fail(LV_ERR_ARG, "NULL server");
  if (!S->cfg.background) {
    for (ServeLane* L : S->lanes) LVTRY(lane_step(S, L));
  }
  std::lock_guard<std::mutex> lock(S->mu);
  if (S->bg_status != LV_OK) return fail(S->bg_status, S->bg_error);
  serve_counts(S, resident, queued);
  return LV_OK;
}

lv_status lv_serve_wait(lv_server* S, uint32_t timeout_ms, int* idle) {
  if (!S) return fail(LV_ERR_ARG, "NULL server");
  std::unique_lock<std::mutex> lk(S->mu);
  auto quiet = [&] {
    uint32_t r = 0, q = 0;
    serve_counts(S, &r, &q);
    return r == 0 && q == 0 && S->busy == 0;
  };
  if (S->cfg.background)
    S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] {
      return !S->finished.empty() || quiet() || S->bg_status != LV_OK;
    });
  if (idle) *idle = quiet() && S->finished.empty() ? 1 : 0;
  if (S->bg_status != LV_OK) return fail(S->bg_status, S->bg_error);
  return LV_OK;
}

lv_status lv_serve_poll(lv_server* S, lv_serve_result* res, uint32_t* assignment, size_t cap,
                        int* got) {
  if (!S || !got) return fail(LV_ERR_ARG, "NULL server or flag");
  *got = 0;
  ServeRequest* r = nullptr;
  {
    std::lock_guard<std::mutex> lock(S->mu);
    if (S->finished.empty()) {
      if (S->bg_status != LV_OK) return fail(S->bg_status, S->bg_error);
      return LV_OK;
    }
    r = S->finished.front();
    if (assignment && cap < r->n) return fail(LV_ERR_ARG, "assignment buffer too small");
    S->finished.pop_front();
  }
  if (res) {
    memset(res, 0, sizeof(*res));
    res->ticket = r->ticket;
    res->modularity = r->q;
    res->n_vertices = r->n;
    res->n_communities = r->n_comm;
    res->levels = r->levels;
    res->lane = r->lane;
    res->submit_ms = r->t_submit;
    res->admit_ms = r->t_admit;
    res->done_ms = r->t_done;
  }
  if (assignment && r->n) memcpy(assignment, r->assignment.data(), r->n * sizeof(uint32_t));
  delete r;
  *got = 1;
  return LV_OK;
}

lv_status lv_serve_get_stats(lv_server* S, lv_serve_stats* out) {
  if (!S || !out) return fail(LV_ERR_ARG, "NULL argument");
  std::lock_guard<std::mutex> lock(S->mu);
  memset(out, 0, sizeof(*out));
  serve_counts(S, &out->resident, &out->queued);
  out->finished = (uint32_t)S->finished.size();
  out->n_lanes = (uint32_t)S->lanes.size();
  for (const ServeLane* L : S->lanes) {
    out->slot_cap += L->slot_cap;
    out->resident_vertices += L->res_n;
    out->resident_entries += L->res_e;
    out->cap_vertices += L->cap_n;
    out->cap_entries += L->cap_e;
    out->steps += L->steps;
    out->admitted += L->admitted;
    out->completed += L->completed;
  }
  out->budget_bytes = S->cfg.budget_bytes;
  return LV_OK;
}

lv_status lv_serve_engine(lv_server* S, uint32_t lane, lv_engine** out) {
  if (!S || !out || lane >= S->lanes.size()) return fail(LV_ERR_ARG, "bad server, lane or out");
  *out = S->lanes[lane]->E;
  return LV_OK;
}

void lv_serve_destroy(lv_server* S) {
  if (!S) return;
  {
    std::lock_guard<std::mutex> lock(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  for (ServeLane* L : S->lanes)
    if (L->worker.joinable()) L->worker.join();
  for (ServeRequest* r : S->finished) delete r;
  for (ServeLane* L : S->lanes) {
    for (ServeRequest* r : L->queue) delete r;
    for (ServeRequest* r : L->by_slot) delete r;
    if (L->E) {
      cudaSetDevice(L->E->device);
      {
        AllocScope alloc_scope(L->E);
        dfree(L->out);
      }
      lv_engine_destroy(L->E);
    }
    if (L->stream) cudaStreamDestroy(L->stream);
    delete L;
  }
  delete S;
}

// ---- autotuning ------------------------------------------------------------
lv_status lv_autotune(lv_engine* E, uint32_t reps, lv_tuning* out) {
  if (E) LVTRY(resolve_pending(E));
  if (!E) return fail(LV_ERR_ARG, "NULL engine");
  if (!E->loaded) return fail(LV_ERR_STATE, "no graph loaded");
  if (E->batch) return fail(LV_ERR_STATE, "a batched run is in progress");
  AllocScope alloc_scope(E);
  cudaSetDevice(E->device);
  if (!reps) reps = 5;
  if (!E->level_ready) LVTRY(prepare_level(E));
  drop_pass_graph(E);  // a captured pass would keep the old kernels
  LVTRY(upload_desc(E, 0.0f));
  const int rule = engine_mode(E);
  lv_tuning t{};
  for (int b = 1; b <= kBuckets; b++) {
    t.bucket_kernel[b] = E->tune[b];
    const uint32_t cnt = E->plan.cls_start[b + 1] - E->plan.cls_start[b];
    if (!cnt) continue;
    // proposals only (no apply), so every launch sees the same state
    float best_ms = 1e30f;
    for (int v = 0; v < KV_COUNT; v++) {
      if (!variant_fits(v, b)) continue;
      uint8_t kv[8];
      memcpy(kv, E->tune, sizeof(kv));
      kv[b] = (uint8_t)v;
      CU(launch_move_bucket(E->d_desc, b, rule, kv, E->st));
      CU(cudaEventRecord(E->ev0, E->st));
      for (uint32_t r = 0; r < reps; r++) CU(launch_move_bucket(E->d_desc, b, rule, kv, E->st));
      CU(cudaEventRecord(E->ev1, E->st));
      CU(cudaEventSynchronize(E->ev1));
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, E->ev0, E->ev1);
      ms /= (float)reps;
      if (ms < best_ms) {
        best_ms = ms;
        t.bucket_kernel[b] = (uint8_t)v;
      }
    }
    t.bucket_ms[b] = best_ms;
    E->tune[b] = t.bucket_kernel[b];
  }
  LVTRY(check_device_error(E));
  if (out) *out = t;
  return LV_OK;
}

lv_status lv_set_tuning(lv_engine* E, const lv_tuning* t) {
  if (!E || !t) return fail(LV_ERR_ARG, "NULL argument");
  for (int b = 1; b <= kBuckets; b++)
    if (!variant_fits(t->bucket_kernel[b], b))
      return fail(LV_ERR_ARG, "kernel variant cannot hold bucket " + std::to_string(b) +
                                  "'s degrees");
  for (int b = 1; b <= kBuckets; b++) E->tune[b] = t->bucket_kernel[b];
  drop_pass_graph(E);
  return LV_OK;
}

lv_status lv_get_tuning(lv_engine* E, lv_tuning* t) {
  if (!E || !t) return fail(LV_ERR_ARG, "NULL argument");
  memset(t, 0, sizeof(*t));
  for (int b = 1; b <= kBuckets; b++) t->bucket_kernel[b] = E->tune[b];
  return LV_OK;
}

lv_status lv_debug_fail_device_alloc(uint64_t n) {
  g_alloc_fail_at.store(0, std::memory_order_relaxed);
  g_alloc_count.store(0, std::memory_order_relaxed);
  g_alloc_fail_at.store(n, std::memory_order_relaxed);
  return LV_OK;
}

lv_status lv_get_sync_count(uint64_t* count) {
  if (!count) return fail(LV_ERR_ARG, "NULL argument");
  *count = sync_count();
  return LV_OK;
}

lv_status lv_get_launch_count(uint64_t* count) {
  if (!count) return fail(LV_ERR_ARG, "NULL argument");
  *count = launch_count();
  return LV_OK;
}

lv_status lv_reset_kernel_stats(lv_engine* E) {
  if (!E) return fail(LV_ERR_ARG, "NULL engine");
  for (int i = 0; i < K_COUNT; i++) E->kst[i] = KStat{};
  return LV_OK;
}

lv_status lv_get_buckets(lv_engine* E, uint8_t* bucket_of, size_t n) {
  if (E) LVTRY(resolve_pending(E));
  AllocScope alloc_scope(E);
  if (!E || (!bucket_of && n)) return fail(LV_ERR_ARG, "NULL argument");
  if (!E->loaded) return fail(LV_ERR_STATE, "no graph loaded");
  if (n != E->n) return fail(LV_ERR_ARG, "buffer length must equal the level's vertex count");
  cudaSetDevice(E->device);
  uint8_t* d = reinterpret_cast<uint8_t*>(E->cb.cursor);
  CU(launch_bucket_ids(E->off(), E->n, d, E->st));
  if (n) CU(cudaMemcpyAsync(bucket_of, d, n, cudaMemcpyDeviceToHost, E->st));
  CU(counted_sync(E->st));
  return LV_OK;
}

}  // extern "C"
