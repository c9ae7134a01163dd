// lv_internal.h -- internal interface between the host engine and the
// sm_100a kernels.  Not part of the C ABI.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace lvb {

// Process-wide count of kernels this library has launched.
void count_launches(unsigned k);
unsigned long long launch_count();
// cudaStreamSynchronize, counted: the host waits for the device this many
// times (process-wide).
cudaError_t counted_sync(cudaStream_t st);
unsigned long long sync_count();

// Move-phase degree buckets (modularity.cu:439): bucket b in 1..7 holds the
// vertices with hi[b-1] < deg <= hi[b]; degree 0 is in no bucket and never
// moves.  Every bucket is one Jacobi step of a pass, in this order.
constexpr int kBuckets = 7;
constexpr uint64_t kBucketHi[kBuckets + 1] = {0, 4, 8, 16, 32, 84, 319,
                                              ~0ull};

// Kernel classes: which kernel processes a vertex.  Classes 1..6 are the
// buckets 1..6; bucket 7 splits into class 7 (shared-memory table, one
// block per vertex) and class 8 (global-memory table, several blocks per
// vertex).  Classes are contiguous in the order array, so bucket 7 is the
// union of classes 7 and 8.
constexpr int kClasses = 9;                 // 0..8, class 0 = degree 0
constexpr uint64_t kHubSmemMaxDeg = 2048;   // class 7 upper degree
constexpr int kHubSmemSlots = 4096;         // table slots of class 7
constexpr uint32_t kHubChunk = 2048;        // edges per block, class 8

__host__ __device__ inline int move_class_of_degree(uint64_t d) {
  return d == 0      ? 0
         : d <= 4    ? 1
         : d <= 8    ? 2
         : d <= 16   ? 3
         : d <= 32   ? 4
         : d <= 84   ? 5
         : d <= 319  ? 6
         : d <= kHubSmemMaxDeg ? 7
                     : 8;
}

// Exclusive scan of one value per thread over a block of whole warps (at
// most 1024 threads); *total receives the block's sum.  `sh` is shared
// scratch of 33 elements.  Every thread of the block must call it.
template <typename T>
__device__ __forceinline__ T block_exclusive_scan(T x, T* sh, T* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = (int)(blockDim.x >> 5);
  T inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) sh[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    const T s = lane < nw ? sh[lane] : T(0);
    T si = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T y = __shfl_up_sync(0xffffffffu, si, o);
      if (lane >= o) si += y;
    }
    sh[lane] = si - s;
    if (lane == 31) sh[32] = si;
  }
  __syncthreads();
  const T r = sh[wid] + inc - x;
  *total = sh[32];
  __syncthreads();  // sh may be reused by the next call
  return r;
}

constexpr uint32_t kEmptyKey = 0xFFFFFFFFu;

// Decision rules, numbered as lv_rule in the C ABI.
constexpr int LV_RULE_PY_I = 0;    // louvian.py:148-151
constexpr int LV_RULE_CUDA_I = 1;  // modularity.cu:182,278,374
// Move mode of the kernels: rule | (gain precision << 1), precision 0 =
// FP32 gains (modularity.cu:149-152), 1 = FP64 gains (louvian.py:135-138).
constexpr int move_mode(int rule, int fp64) { return (rule & 1) | ((fp64 & 1) << 1); }

// Scalars of the current level, resident in device memory so no kernel
// needs a host round trip to learn them.
struct LevelScalars {
  double m64;        // sum_v k_v / 2 (FP64)
  float m;           // FP32 copy used by the gains (modularity.cu:149-152)
  float den;         // 2 * m * m in FP32, evaluated as (2*m)*m
  double q;          // modularity after the most recent sweep
  double intra;      // last sweep's intra-community weight
  double asq;        // last sweep's sum of squared community totals
  uint32_t error;    // set by a kernel when a bounded loop gave up
  uint32_t done_blocks;  // last-block-done counter of reductions
  // device-side pass loop (modularity.cu:466-508 run on the GPU)
  uint32_t passes;       // passes run in the current level
  uint32_t first_fail;   // the first pass gained less than min gain
  double q_prev;         // Q after the previous pass
  double q_before;       // Q before the last pass
  uint32_t any_active;   // some graph's pass loop goes on
  uint32_t act_changed;  // batched form: a graph stopped moving in the last
                         // pass, so the active lists must be compacted again
  double q_start;        // Q when the level's pass loop began
  // single graph: entries of the vertices that moved in the last pass
  // (accumulated by the sweep), and whether the next sweep updates the
  // intra-community weight from those rows only
  unsigned long long moved_acc;
  uint32_t inc_next;
};

// Stop rule evaluated by the modularity sweep's last block when the pass
// loop runs inside a CUDA graph WHILE node.
struct PassControl {
  int enabled;
  int use_handle;             // set the graph condition (WHILE node)
  unsigned long long handle;  // cudaGraphConditionalHandle
  double min_gain;
  uint32_t max_passes;
};

// Per-graph state when a level holds many graphs (batched form): the
// union of the graphs is one block-diagonal CSR and every graph keeps its
// own m, modularity and pass control.
struct GraphState {
  double m_acc;      // sum of k over the graph's vertices (accumulated)
  double m64;        // m = m_acc / 2
  float m;           // FP32 m of the gains
  float den;         // 2 m m in FP32
  double intra_acc;  // modularity sweep accumulators
  double asq_acc;
  double q;          // Q after the latest sweep
  double q_prev;     // Q after the previous pass
  double q_before;   // Q before the last pass
  uint32_t passes;   // passes run at this level
  uint32_t active;   // still moving in this level's pass loop
  uint32_t first_fail;  // first pass gained less than min gain
  uint32_t frozen;   // set by the host: the graph takes no more passes
};

// Batched-form helpers (move.cu).
// gid[v] = graph of vertex v, from the graphs' vertex offsets goff[0..G].
cudaError_t launch_graph_ids(const uint32_t* goff, uint32_t n_graphs, uint32_t n,
                             uint32_t* gid, cudaStream_t st);
// out[i] = asg[i] - base[graph0[i]] for the input vertices whose graph has
// a base (finished now); base[g] == 0xFFFFFFFF leaves out[i] untouched.
cudaError_t launch_finalize_graphs(const uint32_t* asg, size_t n0,
                                   const uint32_t* graph0, const uint32_t* base,
                                   uint32_t* out, cudaStream_t st);
// comm_sz[v] = 0 for the vertices of graphs flagged in drop[] (their
// communities then take no part in the contraction).
cudaError_t launch_drop_graphs(uint32_t* comm_sz, const uint32_t* gid, uint32_t n,
                               const uint32_t* drop, cudaStream_t st);
// out[i] = src[idx[i]]
cudaError_t launch_gather_u32(const uint32_t* src, const uint32_t* idx, uint32_t n,
                              uint32_t* out, cudaStream_t st);

// Read-mostly view of the current level passed to kernels by value.
struct LevelView {
  uint32_t n;
  const uint64_t* __restrict__ off;
  const uint32_t* __restrict__ col;
  const float* __restrict__ w;
  float* k;            // weighted degree (FP32 value of an FP64 row sum)
  uint32_t* comm;      // community of every vertex
  uint32_t* comm_sz;   // vertices per community
  double* tot;         // community totals a_c (FP64, exact for FP32 inputs)
  // second copy of (comm, comm_sz, tot) for passes whose bucket steps apply
  // their own moves (StepIO); equal to the first copy between passes.
  // nullptr where a kernel never needs it.
  uint32_t* comm_alt = nullptr;
  uint32_t* sz_alt = nullptr;
  double* tot_alt = nullptr;
  LevelScalars* sc;
  // batched form only (nullptr for a single graph): graph of every vertex
  // of the level, and the graphs' state
  const uint32_t* gid;
  GraphState* gs;
  uint32_t n_graphs;
};

// Work partition of a level for the "class dispatch" kernels (row sums and
// the modularity sweep): consecutive block ranges serve consecutive classes.
constexpr int kMoveClasses = 7;  // classes 1..7 (class 8, hubs, is never compacted)

// Vertices per dispatch unit (a 256-thread block's share) of classes 1..7:
// G-lane groups for classes 1-4, a warp per vertex for 5-6, a block for 7.
__host__ __device__ constexpr uint32_t class_per_unit(int c) {
  return c <= 4 ? (256u >> (c + 1)) : (c <= 6 ? 8u : 1u);
}

// Class offsets of the vertex order, passed to kernels by value.
struct ClassStarts {
  uint32_t s[kClasses + 1];
};

struct DispatchPlan {
  uint32_t cls_start[kClasses + 1];   // order[] offsets per class
  uint32_t blk_start[kClasses + 1];   // first block of each class (1..8)
  uint32_t hub_count;                 // class 8 vertex count
  uint32_t hub_blocks;                // blocks of class 8 (sum of chunks)
  uint32_t total_blocks;
};

// ---------------------------------------------------------------------------
// scan.cu
// ---------------------------------------------------------------------------
// Scratch for scans of up to `cap` elements.
struct ScanScratch {
  void* buf = nullptr;
  size_t bytes = 0;
};
size_t scan_scratch_bytes(size_t cap);
// Exclusive scans; out may alias in.  When total != nullptr the grand
// total is written there (device pointer).
cudaError_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, size_t n,
                               uint32_t* total, ScanScratch& s,
                               cudaStream_t st);
cudaError_t exclusive_scan_u64(const uint64_t* in, uint64_t* out, size_t n,
                               uint64_t* total, ScanScratch& s,
                               cudaStream_t st);

// Stable partition of [0, n) by vertex degree class: order receives the
// vertices class by class, ascending within a class; cls_count (device,
// kClasses entries) the class sizes.  `tmp` needs partition_tmp_words(n).
size_t partition_tmp_words(size_t n);
cudaError_t partition_by_degree(const uint64_t* off, uint32_t n,
                                uint32_t* order, uint32_t* cls_count,
                                uint32_t* tmp, ScanScratch& s,
                                cudaStream_t st);

// Stable partition of the indices [0, *d_live) into 4 classes by sizes[i]:
// <= lim0, <= lim1, <= lim2, larger.  n_upper bounds *d_live (which is read
// on the device, so no host round trip is needed).
cudaError_t partition_by_size4(const uint64_t* sizes, uint32_t n_upper,
                               const uint32_t* d_live, uint64_t lim0,
                               uint64_t lim1, uint64_t lim2, uint32_t* out,
                               uint32_t* cls_count, uint32_t* tmp,
                               ScanScratch& s, cudaStream_t st);

// ---------------------------------------------------------------------------
// move.cu
// ---------------------------------------------------------------------------
// Row sums k_v, singleton state (comm=id, sizes 1, totals k) and m; with
// rowid the row of every entry, with comm_start comm_start[v] = v.
cudaError_t launch_level_init(const LevelView& L, const uint32_t* order,
                              const DispatchPlan& P, const uint32_t* hub_map,
                              double* partials, uint32_t* rowid, uint32_t* comm_start,
                              cudaStream_t st);
// Modularity of the current state into sc->q (FP64, deterministic).  With
// ctl->enabled the last block also applies the pass stop rule and sets the
// graph condition.
// With act_cnt (batched form) classes 1..7 of `order` are the compacted
// active lists and act_cnt[c] their device-side lengths; every graph's
// modularity then comes from its own vertices' rows and totals.
cudaError_t launch_modularity(const LevelView& L, const uint32_t* order,
                              const DispatchPlan& P, const uint32_t* hub_map,
                              double* partials, cudaStream_t st);

// Hubs (class 8).  A split pass reads every hub row once in chunks of
// kHubChunk entries and writes each chunk's (community, weight) pairs
// grouped by hash partition of the community (partitions of about
// kHubPartKeys distinct communities) into a staging copy of the hub rows;
// entries into the hub's own community are summed there and then.  A merge
// pass runs one block per (hub, partition) over that partition's segment of
// every chunk.  Per hub: the best packed (gain, ~community) key, the
// own-community sums and the plan arrays (fixed for a level).
struct HubArena {
  unsigned long long* best = nullptr;  // [hub_count]
  double* own = nullptr;           // [hub_count] own-community weight w/o self-loop
  double* hot = nullptr;           // [hub_count] own-community weight (all)
  uint32_t* hot_any = nullptr;     // [hub_count] an entry into the own community exists
  uint32_t* nparts = nullptr;      // [hub_count] partitions of the hub
  uint64_t* stage_off = nullptr;   // [hub_count] first staging entry of the hub
  uint64_t* ct_off = nullptr;      // [hub_count] first chunk-table entry of the hub
  uint2* stage = nullptr;          // [hub entries] staged (community, weight bits):
                                   // one 8-byte store and load per entry
  uint32_t* ct = nullptr;          // per hub: chunks x (nparts + 1) segment starts
  uint32_t* blk_vertex = nullptr;  // [units] hub index of each merge unit
  uint32_t* blk_chunk = nullptr;   // [units] partition of the unit
  uint32_t* blk_nchunks = nullptr; // [units] partitions of that hub
  // FP64 gains: every merge unit's best (gain key, ~community), reduced by
  // the decide kernel over the hub's units [unit_start[i], unit_start[i+1])
  unsigned long long* unit_g = nullptr;  // [units]
  uint32_t* unit_c = nullptr;            // [units]
  uint32_t* unit_start = nullptr;        // [hub_count + 1]
  uint32_t units = 0;
};
// Shared table of a hub merge unit (4096 slots, about kHubPartKeys
// communities per partition, load factor ~1/2), and the most partitions a
// hub may have (the split pass keeps one counter per partition in shared
// memory).
constexpr int kHubPartSlots = 4096;
constexpr uint32_t kHubPartKeys = 2048;
constexpr uint32_t kHubMaxParts = 8192;

// Work units of the class-dispatch kernels (row sums, modularity sweep).
struct DispatchArgs {
  DispatchPlan P;
  const uint32_t* order;
  const uint32_t* hub_blk_vertex;
  const uint32_t* hub_blk_chunk;
  double* hub_acc;
  double* partials;         // [2 * gridDim.x]
  const uint32_t* act_cnt;  // batched form: active lengths of classes 1..7
};

// Everything a pass's kernels need about the current level, in device
// memory: the kernels of a pass read it at launch, so one captured pass
// graph serves every level and every run (only this block is rewritten
// between levels), and its grids are fixed.
// Persistent level kernel (single graph): its grid barrier and per-phase
// timers, in device memory, reset before every launch.  Phase kinds are
// numbered as the engine's timing groups: 0..6 the moves of buckets 1..7
// (bucket 7's phase includes the hubs' split pass), 7 the hubs' merge and
// decide passes, 8 apply, 9 the modularity sweep.
constexpr int kPhaseKinds = 10;
struct LevelLoopState {
  unsigned long long arrived;  // barrier arrivals of this launch (monotonic)
  uint32_t abort;              // a barrier wait gave up: every block leaves
  uint32_t timing;             // record per-phase device time
  unsigned long long phase_ns[kPhaseKinds];
  unsigned long long phase_cnt[kPhaseKinds];
};
// LevelScalars::error values: a bounded hash probe gave up / a barrier wait
// of the persistent level kernel gave up.
constexpr uint32_t kErrTableFull = 1u;
constexpr uint32_t kErrBarrierTimeout = 2u;

struct PassDesc {
  LevelView L;
  DispatchArgs A;              // class lists, plan, hub chunks, partials
  uint32_t* prop;              // proposals, parallel to A.order
  const uint32_t* full_order;  // batched form: the uncompacted class lists
  HubArena H;
  // batched form: active lists and their per-graph runs
  uint32_t* act_cnt;
  uint32_t* act_order;
  const uint32_t* cg;
  uint32_t* cg_new;
  uint32_t n_graphs;
  // single graph: the row of every entry (the modularity sweep runs over
  // the entries, not the class lists); nullptr in the batched form
  const uint32_t* rowid;
  uint64_t nnz;
  // device-side pass loop
  double min_gain;
  uint32_t max_passes;
  // persistent level kernel: move kernel variant of every bucket, and its
  // barrier / timer state
  uint8_t tune[8];
  LevelLoopState* loop;
  // persistent level kernel: bucket steps apply their own moves (StepIO)
  // instead of separate apply phases
  uint32_t fused;
  // single graph: every vertex's community when the pass began; nullptr
  // (batched form, lv_config.modularity_full): every sweep is a full one
  uint32_t* comm_start;
};

// How one bucket step of a pass treats the community state.  fused = 0:
// the step only proposes (prop[]), a separate apply launch moves the
// vertices.  fused = 1: the two copies of the state alternate -- the step
// reads copy `parity` (every decision of the bucket against the same
// state: one Jacobi step) and writes its own moves into the other copy,
// which also still lacks the previous step's moves: the step re-applies
// those from prop[] (classes prev_lo..prev_hi; prev_lo = 0: none), so the
// copy it leaves holds every move up to its own.  The pass's modularity
// sweep re-applies the last step's moves, after which both copies are
// equal again.  No apply launch and no grid-wide wait between a bucket's
// decisions and its moves.
struct StepIO {
  int fused;
  int parity;
  int prev_lo;
  int prev_hi;
  // the pass's first step: records every vertex's community in
  // PassDesc::comm_start (the incremental modularity sweep reads it)
  int pass_start;
};

// rowid[j] = the row holding entry j of a CSR of n rows and nnz entries.
cudaError_t launch_row_ids(const uint64_t* off, uint32_t n, uint64_t nnz, uint32_t* rowid,
                           cudaStream_t st);

// Pass kernels: every launch reads the level from D (device memory) and
// uses a fixed grid, so a pass captured once replays on every level.
// passes = 0, first_fail = 0, q_prev = q (start of a level's pass loop),
// for the single graph and for every graph of a batch.
// With ctl->use_handle (single graph) the kernel also sets the WHILE
// node's condition: no pass runs on a level without edge weight.
cudaError_t launch_pass_control_init(const PassDesc* D, const PassControl* ctl, cudaStream_t st);
// Proposals of bucket 1..7 (variant[b]: the kernel, null = defaults), or of
// the hubs (bucket 8); mode = move_mode(rule, fp64 gains).
cudaError_t launch_move_bucket(const PassDesc* D, int bucket, int mode, const uint8_t* variant,
                               cudaStream_t st, StepIO io = StepIO{});
// Applies bucket b's proposals (bucket 7: classes 7 and 8; `compacted`:
// the batched form's active lists, where they are not adjacent).
cudaError_t launch_apply_bucket(const PassDesc* D, int bucket, bool compacted, cudaStream_t st);
// Modularity sweep of the pass; with ctl->enabled also the stop rule
// (limits from D), with ctl->use_handle the WHILE node's condition.
cudaError_t launch_modularity_pass(const PassDesc* D, const PassControl* ctl, cudaStream_t st,
                                   StepIO io = StepIO{});
// The whole pass loop of a single graph's level (modularity.cu:466-508) in
// one cooperative launch of a persistent kernel: every bucket step, apply
// and modularity sweep separated by grid-wide barriers (waits bounded in
// time; a wait that gives up sets kErrBarrierTimeout and ends the kernel),
// the stop rule evaluated identically by every block.  D->loop must be
// zeroed (timing flag aside) before the launch.
cudaError_t launch_level_loop(const PassDesc* D, int mode, cudaStream_t st);
// Blocks of that launch (co-resident: a multiple of the SM count).
unsigned level_loop_grid(int mode);
// Batched form: compacts the class lists to the graphs still moving
// (skipped on the device while no graph stopped in the last pass).
cudaError_t launch_compact_active(const PassDesc* D, cudaStream_t st);
// Blocks of the pass's modularity sweep (its partials need 2 per block).
unsigned pass_dispatch_grid();
// Class-dispatch work units of a level (row sums, modularity sweeps).
DispatchArgs dispatch_args(const uint32_t* order, const DispatchPlan& P, const uint32_t* hub_map,
                           double* partials);
// Proposals for the vertices of kernel class c (1..8; bucket 7 is classes 7
// and 8, both launched before its apply).  proposal[] is parallel to
// order[].
// act_cnt: as for launch_modularity (null: whole classes).
// Move kernel variants a bucket can run on: G-lane groups (one entry per
// lane, degree <= G), a warp with a 128- or 512-slot shared table, a block
// with a 4096-slot table.  All give the same proposals; they differ in how
// the work maps onto the SMs, which the autotuner measures.
enum MoveVariant : uint8_t {
  KV_SMALL4 = 0,
  KV_SMALL8 = 1,
  KV_SMALL16 = 2,
  KV_SMALL32 = 3,
  KV_WARP128 = 4,
  KV_WARP512 = 5,
  KV_BLOCK = 6,
  KV_COUNT = 7
};
// Largest degree a variant handles / a bucket holds (bucket 7: its shared
// table class, degree <= kHubSmemMaxDeg).
constexpr uint64_t variant_max_degree(int v) {
  return v == KV_SMALL4 ? 4 : v == KV_SMALL8 ? 8 : v == KV_SMALL16 ? 16 : v == KV_SMALL32 ? 32
       : v == KV_WARP128 ? 84 : v == KV_WARP512 ? 319 : kHubSmemMaxDeg;
}
constexpr uint64_t bucket_max_degree(int b) {
  return b == 7 ? kHubSmemMaxDeg : kBucketHi[b];
}
constexpr bool variant_fits(int v, int b) {
  return v >= 0 && v < KV_COUNT && b >= 1 && b <= 7 && variant_max_degree(v) >= bucket_max_degree(b);
}
constexpr uint8_t kDefaultVariant[8] = {0, KV_SMALL4, KV_SMALL8, KV_SMALL16, KV_SMALL32,
                                        KV_WARP128, KV_WARP512, KV_BLOCK};

// Batched form.  cg[(c-1)*(G+1) + g] = first index of class c's list
// holding a vertex of graph g (goff: the G+1 graph offsets of the level).
cudaError_t launch_class_graph_starts(const uint32_t* order, const DispatchPlan& P,
                                      const uint32_t* goff, uint32_t G, uint32_t* cg,
                                      cudaStream_t st);
// Compacted lists of classes 1..7 holding only the vertices of graphs
// still active (same class offsets as order), lengths into act_cnt[1..7].

// assignment[i] = map[assignment[i]]
cudaError_t launch_compose(uint32_t* assignment, size_t n0,
                           const uint32_t* map, cudaStream_t st);
// out[i] = map[in[i]]
cudaError_t launch_gather(uint32_t* out, const uint32_t* in, size_t n,
                          const uint32_t* map, cudaStream_t st);
cudaError_t launch_fill_iota(uint32_t* a, size_t n, cudaStream_t st);
// Served form: a[i] = start + i; a[i] = v; a[i] += d.
cudaError_t launch_iota_from(uint32_t* a, size_t n, uint32_t start, cudaStream_t st);
cudaError_t launch_fill_u32(uint32_t* a, size_t n, uint32_t v, cudaStream_t st);
cudaError_t launch_add_u32(uint32_t* a, size_t n, uint32_t d, cudaStream_t st);
cudaError_t launch_add_u64(uint64_t* a, size_t n, uint64_t d, cudaStream_t st);
// Recompute sizes and totals from comm (used when a caller sets comm).
cudaError_t launch_recount(const LevelView& L, cudaStream_t st);
// FP64 modularity of an arbitrary partition (one-off, not hot).
cudaError_t launch_modularity_of(const LevelView& L, const uint32_t* part,
                                 double* tot_scratch, double* out,
                                 cudaStream_t st);
cudaError_t launch_bucket_ids(const uint64_t* off, uint32_t n, uint8_t* out,
                              cudaStream_t st);
unsigned dispatch_grid(const DispatchPlan& P);
// Blocks of the block-per-vertex move kernel resident on the device at once.
unsigned move_block_resident();
unsigned sm_count_cached();
// Opts kernels with more than 48 KB of shared memory in (once per device).
cudaError_t configure_kernels();
cudaError_t configure_contract_kernels();

// ---------------------------------------------------------------------------
// sort.cu
// ---------------------------------------------------------------------------
// Stable LSD radix sort of (key, u32 value) pairs on the low key_bits bits;
// the result is in keys/vals, or in keys_alt/vals_alt when *result_in_alt.
// counts needs radix_sort_scratch_words(n) words, S a scan of that size.
size_t radix_sort_scratch_words(uint64_t n);
template <typename K>
cudaError_t radix_sort_pairs(K* keys, uint32_t* vals, K* keys_alt, uint32_t* vals_alt,
                             uint64_t n, int key_bits, uint32_t* counts, ScanScratch& S,
                             cudaStream_t st, bool* result_in_alt);
// CSR of an edge list with the reference reader's layout (utils.cu:168-229):
// every row in file order, an off-diagonal edge stored in both rows, a
// self-loop once, |w| (1 without weights).  col/wout need room for 2m
// entries; *nnz_host receives the entry count, *bad_host 1 when an index
// is >= n.  Synchronises the stream; scratch is stream-ordered.
cudaError_t csr_from_edges_device(uint32_t n, uint64_t m, const uint32_t* src,
                                  const uint32_t* dst, const float* w, uint64_t* off,
                                  uint32_t* col, float* wout, uint64_t* nnz_host,
                                  uint32_t* bad_host, cudaStream_t st);
// Community listing on the device: out[0..n_comm] the offsets of every
// community's members, out[n_comm + 1 ..] the members (ascending within a
// community).  part[v] < n_comm.
cudaError_t group_by_community(const uint32_t* part, uint32_t n, uint32_t n_comm,
                               uint32_t* out, cudaStream_t st);

// ---------------------------------------------------------------------------
// contract.cu
// ---------------------------------------------------------------------------
struct ContractBuffers {
  uint32_t* flag_id;     // [n] flags -> new ids
  uint32_t* mem_off;     // [n] exclusive scan of comm_sz
  uint32_t* cursor;      // [n]
  uint32_t* members;     // [n] vertices grouped by community
  uint32_t* cnew;        // [n] new id of every vertex's community
  uint64_t* mstart;      // [n+1] flattened edge start of every member
  uint32_t* comm_list;   // [n] old id of every new community
  uint32_t* comm_cls;    // [n] comm_list partitioned by size class
  uint64_t* comm_deg;    // [n] entries per new community
  uint64_t* seg;         // [n] staging offset of every new community's row
  uint64_t* new_deg;     // [n+1] entries per new row -> new offsets
  uint32_t* tcol;        // [E] row staging (cols)
  float* tw;             // [E] row staging (weights)
  uint32_t* tmp;         // partition scratch
  uint32_t* counts;      // [16] device counters
  uint32_t* host_counts; // [16] pinned host mirror (engine-owned)
  uint32_t* keys;        // global tables (class G), u32
  double* vals;          // global tables (class G), FP64
  size_t table_cap;      // slots available in keys/vals
  uint64_t* g_tab_off;   // [cap] per class-G community table offset
  uint32_t* g_tab_size;  // [cap]
  uint32_t* g_blk_comm;  // [cap] per block: index in class-G list
  uint32_t* g_blk_chunk; // [2 cap] per block: chunk, then chunks of its community
  uint32_t* g_blk_first; // [cap + 1] per class-G community: first block
  size_t g_cap;          // entries available in the g_* arrays
};
constexpr uint64_t kMergeWarpMax = 128;    // entries: warp per community
constexpr uint64_t kMergeMidMax = 1024;    // entries: block, 2048-slot table
constexpr uint64_t kMergeBlockMax = 4096;  // entries: block, 8192-slot table
constexpr uint32_t kMergeChunk = 2048;     // entries per block, class G

struct ContractResult {
  uint32_t new_n;
  uint64_t new_nnz;
};
// Buffers of the contraction by sorting (entry-sized, engine-owned).
struct SortBuffers {
  uint64_t* keys[2] = {nullptr, nullptr};  // (new row << bits) | new column
  uint32_t* vals[2] = {nullptr, nullptr};  // entry index
  uint32_t* pos = nullptr;                 // scanned run heads
  uint32_t* counts = nullptr;              // radix digit counts
  ScanScratch scan;                        // scans of entry-sized arrays
  uint64_t cap = 0;                        // entries the buffers hold
};
// Contraction by sorting (single graph): the same new ids, offsets and row
// sets as contract_level, rows sorted by column.  Synchronises the stream
// once at the end.
cudaError_t contract_level_sort(const LevelView& L, uint64_t nnz, ContractBuffers& B,
                                SortBuffers& SB, ScanScratch& S, uint64_t* out_off,
                                uint32_t* out_col, float* out_w, ContractResult* res,
                                cudaStream_t st);
// Contracts level (L, comm) into (out_off, out_col, out_w); writes cnew
// (vertex -> new id) for composing the assignment.  Synchronises the
// stream once for the class sizes (the new vertex count and the plan of the
// multi-block class, built on the device, come with them); with
// defer_total the new entry count is left at B.counts + 8 (u64) for the
// caller's next synchronisation (res->new_nnz = ~0), else it is read with a
// second one.
cudaError_t contract_level(const LevelView& L, uint64_t nnz,
                           ContractBuffers& B, ScanScratch& S,
                           uint64_t* out_off, uint32_t* out_col, float* out_w,
                           ContractResult* res, cudaStream_t st,
                           // host-side growable arena callback
                           cudaError_t (*grow)(void* ctx, size_t slots,
                                               size_t entries),
                           void* grow_ctx, bool defer_total);
// contract_level in two halves around its one synchronisation: the front
// launches everything up to the class sizes and the multi-block plan and
// queues their copy into B.host_counts; the back, called once the stream
// has been synchronised after the front, launches the merges and the new
// CSR.  A caller may put other work and copies between the two and share
// the synchronisation.
cudaError_t contract_front(const LevelView& L, uint64_t nnz, ContractBuffers& B,
                           ScanScratch& S, cudaStream_t st,
                           cudaError_t (*grow)(void* ctx, size_t slots, size_t entries),
                           void* grow_ctx);
cudaError_t contract_back(const LevelView& L, uint64_t nnz, ContractBuffers& B,
                          ScanScratch& S, uint64_t* out_off, uint32_t* out_col,
                          float* out_w, ContractResult* res, cudaStream_t st,
                          cudaError_t (*grow)(void* ctx, size_t slots, size_t entries),
                          void* grow_ctx, bool defer_total);

}  // namespace lvb
