// move.cu -- local-moving phase of one Louvain level on sm_100a.
//
// Reference semantics (upicine/louvain-community-detection):
//   weighted degree k_v ............... modularity.cu:27-49
//   m = sum k / 2 ..................... modularity.cu:457-458
//   singleton state ................... modularity.cu:459-462
//   buckets, one Jacobi step each ..... modularity.cu:439-499
//   isLowerIdx eligibility ............ modularity.cu:85-93
//   gain (FP32) ....................... modularity.cu:149-152
//   argmax, ties -> lower community ... modularity.cu:169-179,359-368
//   decision .......................... louvian.py:148-151 (LV_RULE_PY),
//                                       modularity.cu:182,278,374 (LV_RULE_CUDA)
//   gain arithmetic ................... FP32 as modularity.cu:149-152
//                                       (LV_GAIN_FP32), FP64 as
//                                       louvian.py:135-138 (LV_GAIN_FP64)
//   apply moves + community totals .... modularity.cu:382-398
//   modularity ........................ modularity.cu:400-436
//
// Design (B200-first, not a translation):
//   * Degree classes are computed once per level (degrees do not change
//     within a level) by a stable partition; the reference re-partitions
//     seven times per pass with a host read-back each.
//   * Neighbour-community weights are summed in FP64 (exact for FP32
//     inputs of ordinary dynamic range, hence independent of the order in
//     which concurrent threads add them), then rounded once to FP32 for the
//     gain, which follows the reference expression operation by operation
//     with round-to-nearest intrinsics.
//   * A candidate is evaluated once per distinct neighbour community, and
//     the argmax is a max over packed (gain, ~community) 64-bit keys, so
//     the lowest community id wins ties deterministically.
//   * deg <= 32: G lanes per vertex (G = 4, 8, 16, 32), one edge per lane;
//     equal communities in a group are found with G - 1 shuffles, no hash
//     table at all.  (__match_any_sync costs about one step per distinct
//     value in the warp, and at level 0 all 32 values are distinct.)
//     32 < deg <= 319: one warp per vertex, open-addressing table in shared
//     memory.  319 < deg <= 2048: one block per vertex, 4096-slot shared
//     table.  deg > 2048: one block per (vertex, hash partition of its
//     neighbour communities), 4096-slot shared table, the partitions' best
//     candidates merged with one 64-bit atomicMax each -- no global hash
//     table, whatever the degree.  Shared tables are self-cleaning: a row
//     uses the first slots of its table (a power of two >= 1.5 x its
//     degree), and the candidate scan clears the slots it reads.
//   * Community totals are updated incrementally by the moved vertices
//     only (FP64 atomics), instead of a full recount after every bucket.
#include "lv_internal.h"

#include <algorithm>
#include <cfloat>

namespace lvb {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
// Blocks per SM each pass kernel is compiled for (__launch_bounds__) and
// launched with: the grid-stride kernels run as exactly one resident wave
// (a grid above residency would run a partial second wave of blocks).
constexpr int kSmallPerSM = 8;     // 32 registers
constexpr int kWarp128PerSM = 5;   // 48 registers, 12 KB tables
constexpr int kWarp512PerSM = 4;   // 64 registers, 48 KB tables
constexpr int kBlockPerSM = 3;     // 80 registers, 48 KB table
constexpr int kSplitPerSM = 4;
constexpr int kMergePerSM = 3;     // 80 registers (4 per SM at 64: 9% slower on R-MAT 24)
constexpr int kSweepPerSM = 8;     // apply
constexpr int kModPerSM = 6;       // modularity sweep, 40 registers
static_assert(class_per_unit(1) * 4 == kThreads && class_per_unit(5) == kWarps,
              "dispatch units assume 256-thread blocks");
// shared tables: FP64 values + u32 keys
constexpr int kSlotBytes = 12;
constexpr int kHubPartSmem = kHubPartSlots * kSlotBytes;
constexpr int kBlockTabSmem = kHubSmemSlots * kSlotBytes;

__device__ __forceinline__ unsigned long long umax64(unsigned long long a,
                                                     unsigned long long b) {
  return a > b ? a : b;
}

// Total order on floats mapped to unsigned integers.
__device__ __forceinline__ uint32_t float_key(float f) {
  uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key_float(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}
// max over keys = max gain, then lowest community id.  0 = no candidate.
__device__ __forceinline__ unsigned long long pack_best(float gain,
                                                        uint32_t c) {
  return ((unsigned long long)float_key(gain) << 32) | (uint32_t)(~c);
}

// FP64 gains: the argmax key is the pair (order-preserving bits of the
// double gain, ~community), compared lexicographically -- max gain, then
// lowest community id, as the packed FP32 key.  g == 0: no candidate.
struct Best64 {
  unsigned long long g;
  uint32_t c;
};
__device__ __forceinline__ unsigned long long double_key(double d) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(d);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double key_double(unsigned long long k) {
  return __longlong_as_double(
      (long long)((k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k));
}
// Kernels are instantiated per mode: bit 0 the decision rule, bit 1 the
// gain precision.
template <int MODE>
struct ModeOf {
  static constexpr int kRule = MODE & 1;
  static constexpr int kPrec = MODE >> 1;
};
template <int PREC>
struct BestOf {
  using T = unsigned long long;
};
template <>
struct BestOf<1> {
  using T = Best64;
};
__device__ __forceinline__ unsigned long long best_max(unsigned long long a,
                                                       unsigned long long b) {
  return umax64(a, b);
}
__device__ __forceinline__ Best64 best_max(const Best64& a, const Best64& b) {
  return (a.g > b.g || (a.g == b.g && a.c > b.c)) ? a : b;
}
__device__ __forceinline__ unsigned long long shfl_xor_best(unsigned long long x, int o) {
  return __shfl_xor_sync(0xffffffffu, x, o);
}
__device__ __forceinline__ Best64 shfl_xor_best(const Best64& x, int o) {
  Best64 y;
  y.g = __shfl_xor_sync(0xffffffffu, x.g, o);
  y.c = __shfl_xor_sync(0xffffffffu, x.c, o);
  return y;
}

struct GainCtx {
  float m, den, kv, aown_minus_kv;
  double m64, den64, kv64, aown_minus_kv64;  // FP64 gains
  uint32_t cv, szv;
  bool active;  // the vertex's graph still moves (batched form)
};

// Batched form: a vertex moves only while its graph's pass loop runs.
__device__ __forceinline__ bool vertex_active(const LevelView& L, uint32_t v) {
  return !L.gid || L.gs[L.gid[v]].active;
}

template <int PREC>
__device__ __forceinline__ GainCtx make_ctx(const LevelView& L, uint32_t v,
                                            uint32_t cv) {
  GainCtx g;
  if (L.gid) {
    const GraphState& gs = L.gs[L.gid[v]];
    g.m = gs.m;
    g.den = gs.den;
    g.m64 = gs.m64;
    g.active = gs.active != 0u;
  } else {
    g.m = L.sc->m;
    g.den = L.sc->den;
    g.m64 = L.sc->m64;
    g.active = true;
  }
  g.kv = L.k[v];
  const double acv = L.tot[cv];
  if (PREC) {  // louvian.py:135-138: kv * ((a_own - kv) - a_c) / (2 * (m * m))
    g.kv64 = (double)g.kv;
    g.aown_minus_kv64 = __dsub_rn(acv, g.kv64);
    g.den64 = __dmul_rn(2.0, __dmul_rn(g.m64, g.m64));
  } else {
    g.aown_minus_kv = __fsub_rn((float)acv, g.kv);
  }
  g.cv = cv;
  g.szv = L.comm_sz[cv];
  return g;
}

// (e_c / m) + (k_v * ((a_own - k_v) - a_c) / (2 m m))  -- modularity.cu:149
__device__ __forceinline__ float gain_of(float ec, float ac, const GainCtx& g) {
  float t1 = __fdiv_rn(ec, g.m);
  float t2 = __fsub_rn(g.aown_minus_kv, ac);
  float t3 = __fmul_rn(g.kv, t2);
  float t4 = __fdiv_rn(t3, g.den);
  return __fadd_rn(t1, t4);
}
// The same expression in FP64, operation by operation (louvian.py:135-138).
__device__ __forceinline__ double gain_of64(double ec, double ac, const GainCtx& g) {
  const double t1 = __ddiv_rn(ec, g.m64);
  const double t2 = __dsub_rn(g.aown_minus_kv64, ac);
  const double t3 = __dmul_rn(g.kv64, t2);
  const double t4 = __ddiv_rn(t3, g.den64);
  return __dadd_rn(t1, t4);
}

// Candidate key of neighbour community c (summed weight ec, total ac, size
// szc); none if c is not eligible under isLowerIdx (modularity.cu:85-93).
template <int PREC>
__device__ __forceinline__ typename BestOf<PREC>::T candidate_loaded(const GainCtx& g,
                                                                     uint32_t c, double ec,
                                                                     uint32_t szc, double ac) {
  using K = typename BestOf<PREC>::T;
  if (g.szv == 1 && szc == 1 && !(c < g.cv)) return K{};
  if constexpr (PREC) {
    return Best64{double_key(gain_of64(ec, ac, g)), ~c};
  } else {
    return pack_best(gain_of((float)ec, (float)ac, g), c);
  }
}

// Size of candidate community c as candidate_loaded needs it: only a
// singleton vertex tests the candidate's size, and only for c > cv
// (isLowerIdx), so every other candidate skips the gather -- these
// per-lane random loads are what the move kernels' L1 pipe spends its
// cycles on.
__device__ __forceinline__ uint32_t candidate_size(const LevelView& L, const GainCtx& g,
                                                   uint32_t c) {
  if (c == g.cv) return g.szv;
  return (g.szv == 1u && c > g.cv) ? L.comm_sz[c] : 0u;
}

template <int PREC>
__device__ __forceinline__ typename BestOf<PREC>::T candidate(const LevelView& L,
                                                              const GainCtx& g, uint32_t c,
                                                              double ec) {
  return candidate_loaded<PREC>(g, c, ec, candidate_size(L, g, c), L.tot[c]);
}

template <int RULE>
__device__ __forceinline__ uint32_t decide(unsigned long long best, double own,
                                           const GainCtx& g) {
  if (best == 0ull || !g.active) return g.cv;
  const float bg = key_float((uint32_t)(best >> 32));
  const uint32_t bc = ~(uint32_t)best;
  bool move;
  if (RULE == LV_RULE_CUDA_I) {
    move = __fsub_rn(bg, __fdiv_rn((float)own, g.m)) > 0.0f;
  } else {
    move = bg > 0.0f;
  }
  return move ? bc : g.cv;
}
template <int RULE>
__device__ __forceinline__ uint32_t decide(const Best64& best, double own, const GainCtx& g) {
  if (best.g == 0ull || !g.active) return g.cv;
  const double bg = key_double(best.g);
  const uint32_t bc = ~best.c;
  bool move;
  if (RULE == LV_RULE_CUDA_I) {  // max_gain - e_own / m > 0 in FP64
    move = __dsub_rn(bg, __ddiv_rn(own, g.m64)) > 0.0;
  } else {
    move = bg > 0.0;
  }
  return move ? bc : g.cv;
}

template <int G, class K>
__device__ __forceinline__ K group_max(K x) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) x = best_max(x, shfl_xor_best(x, o));
  return x;
}
template <int G>
__device__ __forceinline__ double group_sum(double x) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
  return x;
}

// Batched form: adds every lane's val into gs[key].*field with one atomic
// per run of equal keys.  Called by all 32 lanes; keys must be
// non-decreasing across the lanes (vertex ids ascend within a class order,
// and graphs own contiguous id ranges), a lane without a value passes
// kNoGraph.  A segmented suffix sum leaves each run's total in its first
// lane.
constexpr uint32_t kNoGraph = 0xFFFFFFFFu;
using GraphField = double GraphState::*;
__device__ __forceinline__ void warp_graph_add(GraphState* gs, GraphField field, uint32_t key,
                                               double val) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double ov = __shfl_down_sync(kFull, val, o);
    const uint32_t ok = __shfl_down_sync(kFull, key, o);
    if (lane + o < 32 && ok == key) val += ov;
  }
  const uint32_t pk = __shfl_up_sync(kFull, key, 1);
  if (key != kNoGraph && (lane == 0 || pk != key) && val != 0.0)
    atomicAdd(&(gs[key].*field), val);
}

// Open addressing with linear probing.  Probe counts are bounded by the
// table size; a full table (impossible while a table holds more slots than
// the row has entries) sets the error flag.
// Slot from the top bits of a multiplicative (Fibonacci) hash: the low bits
// of key * odd depend only on the key's low bits, and vertex ids such as
// R-MAT's share low-bit patterns, which piled them into a few probe chains.
__device__ __forceinline__ uint32_t hash_slot(uint32_t key, uint32_t mask) {
  return __umulhi(key * 2654435761u, mask + 1u);  // mask + 1: a power of two
}
// Table slots used for a row of d entries: a power of two >= 1.5 d (load
// factor <= 2/3), at most tmax (the class's shared-memory table).
__device__ __forceinline__ uint32_t table_size_for(uint32_t d, uint32_t tmax) {
  const uint32_t want = d + (d >> 1) + 1;
  uint32_t t = 32;
  while (t < want) t <<= 1;
  return t < tmax ? t : tmax;
}

// Slot of key in a shared table of mask + 1 slots (inserted if absent).
// The table is cleared in full once, when a warp or block starts; after a
// row, the candidate scan (scan_table_and_clear) empties the slots it used.
// No shared counter: keeping a list of taken slots cost one same-address
// atomic per distinct key, which serialised whole warps.
__device__ __forceinline__ uint32_t table_insert(uint32_t* keys, uint32_t mask,
                                                 uint32_t key, LevelScalars* sc) {
  uint32_t h = hash_slot(key, mask);
  for (uint32_t it = 0; it <= mask; it++) {
    uint32_t cur = keys[h];
    if (cur == key) return h;
    if (cur == kEmptyKey) {
      uint32_t prev = atomicCAS(&keys[h], kEmptyKey, key);
      if (prev == kEmptyKey || prev == key) return h;
    }
    h = (h + 1) & mask;
  }
  atomicExch(&sc->error, 1u);
  return 0;
}

// table_insert that also reports whether this call put the key into the
// table: that thread owns the key's candidate (exactly one per distinct
// key), evaluates it once the table is complete and empties its slot.
__device__ __forceinline__ uint32_t table_claim(uint32_t* keys, uint32_t mask, uint32_t key,
                                                LevelScalars* sc, bool& claimed) {
  uint32_t h = hash_slot(key, mask);
  claimed = false;
  for (uint32_t it = 0; it <= mask; it++) {
    uint32_t cur = keys[h];
    if (cur == key) return h;
    if (cur == kEmptyKey) {
      const uint32_t prev = atomicCAS(&keys[h], kEmptyKey, key);
      if (prev == kEmptyKey) {
        claimed = true;
        return h;
      }
      if (prev == key) return h;
    }
    h = (h + 1) & mask;
  }
  atomicExch(&sc->error, 1u);
  return 0;
}

// Adds each lane's (key, w) to a shared table, the lanes holding the same
// key as the wave's first entry summed with shuffles into one atomic: in
// late passes a hub's neighbours crowd into a few communities, and
// hundreds of threads looping on one slot's FP64 compare-and-swap made the
// merge slower pass after pass.  A wave of distinct keys pays two ballots.
__device__ __forceinline__ void table_add_wave(uint32_t* keys, double* vals, uint32_t mask,
                                               bool has, uint32_t key, double w,
                                               LevelScalars* sc) {
  const int lane = threadIdx.x & 31;
  const unsigned hm = __ballot_sync(0xffffffffu, has);
  if (!hm) return;  // warp-uniform
  const int lead = __ffs(hm) - 1;
  const uint32_t kl = __shfl_sync(0xffffffffu, key, lead);
  const unsigned m = __ballot_sync(0xffffffffu, has && key == kl);
  if (__popc(m) > 1) {  // warp-uniform
    double x = (m >> lane & 1u) ? w : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == lead) atomicAdd(&vals[table_insert(keys, mask, kl, sc)], x);
    if (m >> lane & 1u) return;
  }
  if (has) atomicAdd(&vals[table_insert(keys, mask, key, sc)], w);
}

// ---------------------------------------------------------------------------
// Community state of a bucket step (StepIO).  step_view's comm / comm_sz /
// tot are the copy the step reads; a fused step writes its moves into the
// other copy (write_copy), fetched from the descriptor where a move is
// recorded rather than kept in registers through the step.
// ---------------------------------------------------------------------------
__device__ __forceinline__ LevelView step_view(const PassDesc* __restrict__ D, const StepIO& io) {
  LevelView L = D->L;
  if (io.parity) {
    L.comm = D->L.comm_alt;
    L.comm_sz = D->L.sz_alt;
    L.tot = D->L.tot_alt;
  }
  return L;
}

struct StateCopy {
  uint32_t* comm;
  uint32_t* sz;
  double* tot;
};
__device__ __forceinline__ StateCopy write_copy(const PassDesc* __restrict__ D,
                                                const StepIO& io) {
  return io.parity ? StateCopy{D->L.comm, D->L.comm_sz, D->L.tot}
                   : StateCopy{D->L.comm_alt, D->L.sz_alt, D->L.tot_alt};
}

// assignCommunity + incremental totals (modularity.cu:382-398) of one
// vertex of weighted degree kv moving from oc to nc, into copy W.  FP64
// sums of FP32 degrees are exact, so the order of the atomics does not
// matter.
__device__ __forceinline__ void move_into(const StateCopy& W, uint32_t v, float kv, uint32_t oc,
                                          uint32_t nc) {
  atomicSub(&W.sz[oc], 1u);
  atomicAdd(&W.sz[nc], 1u);
  atomicAdd(&W.tot[oc], -(double)kv);
  atomicAdd(&W.tot[nc], (double)kv);
  W.comm[v] = nc;
}

// The previous step's moves into the written copy: a vertex of classes
// prev_lo..prev_hi still has its old community there (it moves in no
// other step of the pass), its proposal is in prop[].
__device__ __forceinline__ void reapply_prev_step(const PassDesc* __restrict__ D,
                                                  const StepIO& io, uint32_t bid,
                                                  uint32_t nblk) {
  if (!io.fused || io.prev_lo == 0) return;
  const StateCopy W = write_copy(D, io);
  const float* __restrict__ k = D->L.k;
  for (int c = io.prev_lo; c <= io.prev_hi; c++) {
    const uint32_t s0 = D->A.P.cls_start[c];
    const uint32_t count = (D->act_cnt && c <= kMoveClasses) ? D->act_cnt[c]
                                                             : D->A.P.cls_start[c + 1] - s0;
    const uint32_t* __restrict__ verts = D->A.order + s0;
    const uint32_t* prop = D->prop + s0;
    for (uint32_t i = bid * blockDim.x + threadIdx.x; i < count; i += nblk * blockDim.x) {
      const uint32_t v = verts[i];
      const uint32_t nc = prop[i];
      const uint32_t oc = W.comm[v];
      if (nc != oc) move_into(W, v, k[v], oc, nc);
    }
  }
}

// A vertex of a class list with its row bounds and community: the block-
// per-vertex kernel loads the next vertex's while it works on the current
// one, so its id -> offsets -> community chain is off the critical path.
struct VertexRow {
  uint32_t v;
  uint64_t s, e;
  uint32_t cv;
};
__device__ __forceinline__ VertexRow fetch_vertex(const LevelView& L,
                                                  const uint32_t* __restrict__ verts,
                                                  uint32_t vidx, uint32_t count) {
  VertexRow r{0u, 0ull, 0ull, 0u};
  if (vidx < count) {
    r.v = verts[vidx];
    r.s = L.off[r.v];
    r.e = L.off[r.v + 1];
    r.cv = L.comm[r.v];
  }
  return r;
}

// The pass's first step records every vertex's community (both copies of
// the state are equal then) for the incremental modularity sweep.
__device__ __forceinline__ void record_pass_start(const PassDesc* __restrict__ D,
                                                  const LevelView& L, const StepIO& io,
                                                  uint32_t bid, uint32_t nblk) {
  uint32_t* cs = D->comm_start;
  if (!io.pass_start || !cs) return;
  for (uint32_t v = bid * blockDim.x + threadIdx.x; v < L.n; v += nblk * blockDim.x) {
    const uint32_t c = L.comm[v];
    if (cs[v] != c) cs[v] = c;
  }
}

// Records a decision: the proposal (read by the next step's re-apply and
// by the separate apply launch) and, in a fused step, the move itself.
__device__ __forceinline__ void record_decision(const PassDesc* __restrict__ D,
                                                const StepIO& io, uint32_t* prop_slot,
                                                uint32_t v, const GainCtx& g, uint32_t nc) {
  *prop_slot = nc;
  if (io.fused && nc != g.cv) move_into(write_copy(D, io), v, g.kv, g.cv, nc);
}

// ---------------------------------------------------------------------------
// Move kernels
// ---------------------------------------------------------------------------

// Every kernel body below takes its block's index and the number of blocks
// sharing the work (a grid-stride loop over work units), and its shared
// memory from the caller: the standalone kernels pass blockIdx/gridDim and
// their own shared arrays, the persistent level kernel the same body with
// its one shared-memory arena.
template <int G, int MODE>
__device__ __forceinline__ void small_body(const PassDesc* __restrict__ D, int cls,
                                           uint32_t bid, uint32_t nblk, double (*sums)[32],
                                           const StepIO io = StepIO{}) {
  constexpr int RULE = ModeOf<MODE>::kRule, PREC = ModeOf<MODE>::kPrec;
  using K = typename BestOf<PREC>::T;
  const LevelView L = step_view(D, io);
  reapply_prev_step(D, io, bid, nblk);
  record_pass_start(D, L, io, bid, nblk);
  const uint32_t s0 = D->A.P.cls_start[cls];
  const uint32_t* __restrict__ verts = D->A.order + s0;
  uint32_t* __restrict__ prop = D->prop + s0;
  // batched form: the class's active vertices
  const uint32_t count = D->act_cnt ? D->act_cnt[cls] : D->A.P.cls_start[cls + 1] - s0;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int gl = lane & (G - 1);
  const uint32_t per_block = kThreads / G;
  for (uint32_t base = bid * per_block; base < count; base += nblk * per_block) {
    const uint32_t vidx = base + threadIdx.x / G;
    const bool vvalid = vidx < count;
    uint32_t v = 0, d = 0, cv = 0;
    uint64_t s = 0;
    bool act = false;
    if (vvalid) {
      v = verts[vidx];
      s = L.off[v];
      d = (uint32_t)(L.off[v + 1] - s);
      cv = L.comm[v];
      act = vertex_active(L, v);
    }
    const bool has = act && gl < (int)d;
    // the vertex's own state is read alongside its row (no dependency)
    GainCtx g;
    if (vvalid) g = make_ctx<PREC>(L, v, cv);
    uint32_t u = 0, cu = 0, szc = 0;
    float wt = 0.0f;
    double ac = 0.0;
    if (has) {
      u = L.col[s + gl];
      wt = L.w[s + gl];
      cu = L.comm[u];
      szc = candidate_size(L, g, cu);  // the candidate's data, read before the grouping
      ac = L.tot[cu];
    }
    // the own community's entries are summed with shuffles (its lowest
    // lane holds the sum); the others through one shared slot per distinct
    // community
    const bool is_hot = has && cu == cv;
    const bool ins = has && !is_hot;
    const double hv = group_sum<G>(is_hot ? (double)wt : 0.0);
    const unsigned gmask = (G == 32) ? kFull : (((1u << G) - 1u) << (lane & ~(G - 1)));
    const unsigned hmask = __ballot_sync(kFull, is_hot) & gmask;
    const int hot_leader = hmask ? __ffs(hmask) - 1 : -1;
    // leader of an entry: the group's lowest lane holding the same community
    const uint32_t gbase = lane & ~(G - 1);
    const uint32_t mykey = ins ? cu : kEmptyKey;
    uint32_t first = gl;
#pragma unroll
    for (int o = 1; o < G; o++) {
      const uint32_t src = (gl + o) & (G - 1);
      const uint32_t ok = __shfl_sync(kFull, mykey, gbase | src);
      if (ins && ok == cu && src < first) first = src;
    }
    const int leader = (int)(gbase | first);
    sums[wib][lane] = (lane == hot_leader) ? hv : 0.0;
    __syncwarp();
    if (ins) atomicAdd(&sums[wib][leader], (double)wt);
    double own = 0.0;
    if (RULE == LV_RULE_CUDA_I && is_hot && u != v) own = (double)wt;
    __syncwarp();
    K best{};
    if ((ins && leader == lane) || lane == hot_leader)
      best = candidate_loaded<PREC>(g, cu, sums[wib][lane], szc, ac);
    best = group_max<G>(best);
    if (RULE == LV_RULE_CUDA_I) own = group_sum<G>(own);
    if (vvalid && gl == 0) record_decision(D, io, &prop[vidx], v, g, decide<RULE>(best, own, g));
    __syncwarp();
  }
}

// deg <= G: G lanes per vertex, one edge per lane.
template <int G, int MODE>
__global__ void __launch_bounds__(kThreads, kSmallPerSM)
    move_small_kernel(const PassDesc* __restrict__ D, int cls, StepIO io) {
  __shared__ double sums[kWarps][32];
  small_body<G, MODE>(D, cls, blockIdx.x, gridDim.x, sums, io);
}

// Best candidate among the taken slots of the first tv slots (nthr
// threads from tid, four slots per thread at a time so the gathers
// overlap); each thread empties the taken slots it read, leaving the table
// clean.
template <int PREC, bool kAllSizes = false>
__device__ __forceinline__ typename BestOf<PREC>::T scan_table_and_clear(
    const LevelView& L, const GainCtx& g, uint32_t* keys, double* vals,
    uint32_t tv, uint32_t tid, uint32_t nthr) {
  typename BestOf<PREC>::T best{};
#pragma unroll 1
  for (uint32_t i0 = tid; i0 < tv; i0 += 4 * nthr) {
    uint32_t c[4], szc[4];
    double ec[4], ac[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const uint32_t i = i0 + q * nthr;
      c[q] = i < tv ? keys[i] : kEmptyKey;
      ec[q] = c[q] != kEmptyKey ? vals[i] : 0.0;
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      if (c[q] != kEmptyKey) {
        // kAllSizes: every candidate's size, loaded with its total (the hub
        // merge, 7% faster on R-MAT 24 than gathering only the sizes the
        // isLowerIdx test reads, which it does after its segment walk)
        szc[q] = kAllSizes ? L.comm_sz[c[q]] : candidate_size(L, g, c[q]);
        ac[q] = L.tot[c[q]];
      }
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      if (c[q] != kEmptyKey) {
        best = best_max(best, candidate_loaded<PREC>(g, c[q], ec[q], szc[q], ac[q]));
        const uint32_t i = i0 + q * nthr;
        keys[i] = kEmptyKey;
        vals[i] = 0.0;
      }
    }
  }
  return best;
}

// Row entries [s, e_end) spread over NT threads as 4-entry vectors: thread
// t holds slot i = 4 k + j, the entry at 4 (s / 4 + k NT + t) + j (k < NV),
// when it falls in the row.  A vector entirely inside the row is one
// 128-bit load of columns and one of weights (vec_ok: both arrays 16-byte
// aligned, as every buffer the engine allocates); the vectors at the row's
// ends are loaded entry by entry, so nothing outside the row is read.
// Slots outside the row get column `fill` and weight 0.
template <int NV, int NT>
__device__ __forceinline__ uint64_t vec_entry(uint64_t s, uint32_t t, int i) {
  return ((s >> 2) + (uint64_t)(i >> 2) * NT + t) * 4 + (uint64_t)(i & 3);
}
template <int NV, int NT>
__device__ __forceinline__ void load_row_vec(const LevelView& L, uint64_t s, uint64_t e_end,
                                             uint32_t t, uint32_t fill, bool vec_ok,
                                             uint32_t (&cu)[4 * NV], float (&wt)[4 * NV]) {
#pragma unroll
  for (int k = 0; k < NV; k++) {
    const uint64_t base = vec_entry<NV, NT>(s, t, 4 * k);
    if (vec_ok && base >= s && base + 4 <= e_end) {
      const uint4 c = __ldg(reinterpret_cast<const uint4*>(L.col) + (base >> 2));
      const float4 w = __ldg(reinterpret_cast<const float4*>(L.w) + (base >> 2));
      cu[4 * k] = c.x;
      cu[4 * k + 1] = c.y;
      cu[4 * k + 2] = c.z;
      cu[4 * k + 3] = c.w;
      wt[4 * k] = w.x;
      wt[4 * k + 1] = w.y;
      wt[4 * k + 2] = w.z;
      wt[4 * k + 3] = w.w;
    } else {
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const uint64_t idx = base + (uint64_t)j;
        const bool in = idx >= s && idx < e_end;
        cu[4 * k + j] = in ? L.col[idx] : fill;
        wt[4 * k + j] = in ? L.w[idx] : 0.0f;
      }
    }
  }
}

// The candidates of the keys a thread claimed while its entries went into
// a complete table: entry slot i's table slot is the i-th 16-bit field of
// `slots` (bit i of `owned` set); the key is read back from the table, so
// the entries' registers are free once they are inserted.  Four at a time,
// so their gathers overlap; each slot is emptied after it is read, which
// leaves the table clean without a scan of its empty slots.
template <int NE>
__device__ __forceinline__ void claim_slot(uint32_t (&slots)[(NE + 1) / 2], uint32_t& owned,
                                           int i, uint32_t slot) {
  owned |= 1u << i;
#pragma unroll
  for (int j = 0; j < (NE + 1) / 2; j++)  // i is a constant of the unrolled caller
    if (j == (i >> 1)) slots[j] |= slot << (16 * (i & 1));
}
template <int PREC, int NE>
__device__ __forceinline__ typename BestOf<PREC>::T eval_owned(
    const LevelView& L, const GainCtx& g, uint32_t* keys, double* vals,
    const uint32_t (&slots)[(NE + 1) / 2], uint32_t owned, typename BestOf<PREC>::T best) {
#pragma unroll
  for (int i0 = 0; i0 < NE; i0 += 4) {
    if (((owned >> i0) & 0xFu) == 0u) continue;
    uint32_t szc[4], slot[4], c[4];
    double ec[4], ac[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = i0 + q;
      if (i < NE && (owned >> i & 1u)) {
        slot[q] = (slots[i >> 1] >> (16 * (i & 1))) & 0xFFFFu;
        c[q] = keys[slot[q]];
        ec[q] = vals[slot[q]];
        szc[q] = candidate_size(L, g, c[q]);
        ac[q] = L.tot[c[q]];
      }
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = i0 + q;
      if (i < NE && (owned >> i & 1u)) {
        best = best_max(best, candidate_loaded<PREC>(g, c[q], ec[q], szc[q], ac[q]));
        keys[slot[q]] = kEmptyKey;
        vals[slot[q]] = 0.0;
      }
    }
  }
  return best;
}

// The own community's candidate, for the thread that claimed its slot.
template <int PREC>
__device__ __forceinline__ typename BestOf<PREC>::T eval_own_slot(
    const LevelView& L, const GainCtx& g, uint32_t* keys, double* vals, uint32_t slot,
    typename BestOf<PREC>::T best) {
  const double ec = vals[slot];
  best = best_max(best, candidate_loaded<PREC>(g, g.cv, ec, g.szv, L.tot[g.cv]));
  keys[slot] = kEmptyKey;
  vals[slot] = 0.0;
  return best;
}

// 32 < deg <= 319: one warp per vertex, T-slot table per warp.  All of a
// row's loads (at most MAXW waves of 32) are issued before any insertion,
// so a vertex costs one memory latency chain instead of one per wave.
template <int T, int MAXW, int MODE>
__device__ __forceinline__ void warp_body(const PassDesc* __restrict__ D, int cls, uint32_t bid,
                                          uint32_t nblk, unsigned char* smem_raw,
                                          const StepIO io = StepIO{}) {
  constexpr int RULE = ModeOf<MODE>::kRule, PREC = ModeOf<MODE>::kPrec;
  const LevelView L = step_view(D, io);
  reapply_prev_step(D, io, bid, nblk);
  record_pass_start(D, L, io, bid, nblk);
  const uint32_t s0 = D->A.P.cls_start[cls];
  const uint32_t* __restrict__ verts = D->A.order + s0;
  uint32_t* __restrict__ prop = D->prop + s0;
  const uint32_t count = D->act_cnt ? D->act_cnt[cls] : D->A.P.cls_start[cls + 1] - s0;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double* vals = reinterpret_cast<double*>(smem_raw) + wib * T;
  uint32_t* keys =
      reinterpret_cast<uint32_t*>(smem_raw + sizeof(double) * T * kWarps) + wib * T;
  uint32_t clean = 0;  // leading table slots known to be empty
  const bool vec_ok = (((uintptr_t)L.col | (uintptr_t)L.w) & 15u) == 0;
  for (uint32_t vidx = bid * kWarps + wib; vidx < count; vidx += nblk * kWarps) {
    const uint32_t v = verts[vidx];
    const uint64_t s = L.off[v];
    const uint32_t d = (uint32_t)(L.off[v + 1] - s);
    const uint32_t cv = L.comm[v];
    if (!vertex_active(L, v)) {  // warp-uniform: one vertex per warp
      if (lane == 0) prop[vidx] = cv;
      continue;
    }
    const uint32_t tv = table_size_for(d, T);
    if (tv > clean) {  // warp-uniform; the scan empties what a row used
      for (uint32_t i = clean + lane; i < tv; i += 32) {
        keys[i] = kEmptyKey;
        vals[i] = 0.0;
      }
      clean = tv;
      __syncwarp();
    }
    const GainCtx g = make_ctx<PREC>(L, v, cv);
    // every load of the row issued before any is used.  Rows of up to 319
    // entries come in 4-entry vectors (a vector crossing the row's start or
    // end takes one extra slot): 5% faster on R-MAT 24's bucket 6; the
    // shorter rows of the 128-slot variant keep one entry per lane per wave
    // (vectors made it spill and run 17% slower there)
    constexpr bool kVec = MAXW >= 8;
    constexpr int NV = kVec ? (8 * MAXW + 1 + 31) / 32 : 0;
    constexpr int NE = kVec ? 4 * NV : MAXW;
    static_assert(NE <= 32, "one self-loop bit per slot");
    uint32_t cu[NE];
    float wt[NE];
    const uint64_t e_end = s + d;
    // absolute entry index of slot i of this lane
    auto entry_of = [&](int i, uint32_t ln) -> uint64_t {
      return kVec ? vec_entry<NV, 32>(s, ln, i) : s + (uint64_t)i * 32 + ln;
    };
    if constexpr (kVec) {
      load_row_vec<NV, 32>(L, s, e_end, lane, v, vec_ok, cu, wt);
    } else {
#pragma unroll
      for (int i = 0; i < NE; i++) {
        const uint64_t idx = entry_of(i, lane);
        cu[i] = idx < e_end ? L.col[idx] : v;
        wt[i] = idx < e_end ? L.w[idx] : 0.0f;
      }
    }
    unsigned self_mask = 0u;  // slots whose entry is the self-loop
#pragma unroll
    for (int i = 0; i < NE; i++) {
      const uint64_t idx = entry_of(i, lane);
      const bool has = idx >= s && idx < e_end;
      if (has && cu[i] == v) self_mask |= 1u << i;
      cu[i] = has ? L.comm[cu[i]] : kEmptyKey;  // kEmptyKey: no entry
    }
    double own = 0.0, hot = 0.0;
    bool hot_seen = false;
#pragma unroll
    for (int i = 0; i < NE; i++) {
      if ((!kVec || (i & 3) == 0) && entry_of(i, 0) >= e_end) break;  // warp-uniform
      const bool has = cu[i] != kEmptyKey;
      // entries into the vertex's own community (most of them once moves
      // converge) are summed in registers, not in one contended slot
      const bool is_hot = has && cu[i] == cv;
      const bool ins = has && !is_hot;
      if (is_hot) {
        hot += (double)wt[i];
        hot_seen = true;
        if (RULE == LV_RULE_CUDA_I && !(self_mask >> i & 1u)) own += (double)wt[i];
      }
      // every lane inserts its own entry: equal keys meet in the CAS
      if (ins) atomicAdd(&vals[table_insert(keys, tv - 1, cu[i], L.sc)], (double)wt[i]);
    }
    hot = group_sum<32>(hot);
    if (__any_sync(kFull, hot_seen) && lane == 0) {
      const uint32_t slot = table_insert(keys, tv - 1, cv, L.sc);
      vals[slot] += hot;
    }
    __syncwarp();
    // a scan of the row's table range: owner evaluation as in the block
    // kernel made this kernel spill and run 37% slower at R-MAT 24, and a
    // list of the claimed slots (a ballot per wave) 38% slower
    auto best = scan_table_and_clear<PREC>(L, g, keys, vals, tv, lane, 32);
    best = group_max<32>(best);
    if (RULE == LV_RULE_CUDA_I) own = group_sum<32>(own);
    if (lane == 0) record_decision(D, io, &prop[vidx], v, g, decide<RULE>(best, own, g));
    __syncwarp();
  }
}

template <int T, int MAXW, int MODE>
__global__ void __launch_bounds__(kThreads, T == 128 ? kWarp128PerSM : kWarp512PerSM)
    move_warp_kernel(const PassDesc* __restrict__ D, int cls, StepIO io) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  warp_body<T, MAXW, MODE>(D, cls, blockIdx.x, gridDim.x, smem_raw, io);
}

template <class K>
__device__ __forceinline__ K block_max(K x, K* red) {
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  x = group_max<32>(x);
  if (lane == 0) red[wib] = x;
  __syncthreads();
  K r{};
  if (threadIdx.x == 0) {
    for (int i = 0; i < kWarps; i++) r = best_max(r, red[i]);
  }
  __syncthreads();
  return r;  // valid in thread 0
}

__device__ __forceinline__ double block_sum(double x, double* red) {
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  x = group_sum<32>(x);
  if (lane == 0) red[wib] = x;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < kWarps; i++) r += red[i];
  }
  __syncthreads();
  return r;  // valid in thread 0
}

// Loads entries [lo, end) of row s (at most MAXW waves of the block) into
// registers -- every load issued before any is used -- then inserts them
// into a table (clear it before, synchronise after).  cu / wt / owned come
// back as eval_owned reads them.
template <int MAXW, int RULE>
__device__ __forceinline__ void insert_block_range(const LevelView& L, uint64_t s,
                                                   uint64_t lo, uint64_t end,
                                                   uint32_t v, uint32_t cv,
                                                   uint32_t* keys, double* vals,
                                                   uint32_t mask, double& own,
                                                   double& hot, bool& hot_seen,
                                                   uint32_t (&slots)[(MAXW + 1) / 2],
                                                   uint32_t& owned) {
  uint32_t cu[MAXW];
  float wt[MAXW];
  unsigned self_mask = 0u;
  owned = 0u;
#pragma unroll
  for (int k = 0; k < MAXW; k++) {
    const uint64_t j = lo + (uint64_t)k * kThreads + threadIdx.x;
    cu[k] = v;
    wt[k] = 0.0f;
    if (j < end) {
      cu[k] = L.col[s + j];
      wt[k] = L.w[s + j];
    }
  }
#pragma unroll
  for (int k = 0; k < MAXW; k++) {
    const uint64_t j = lo + (uint64_t)k * kThreads + threadIdx.x;
    if (cu[k] == v) self_mask |= 1u << k;
    cu[k] = (j < end) ? L.comm[cu[k]] : kEmptyKey;
  }
#pragma unroll
  for (int k = 0; k < MAXW; k++) {
    if (lo + (uint64_t)k * kThreads >= end) break;  // block-uniform
    const bool has = lo + (uint64_t)k * kThreads + threadIdx.x < end;
    // own-community entries go to the caller's register sum (hot)
    const bool is_hot = has && cu[k] == cv;
    const bool ins = has && !is_hot;
    if (is_hot) {
      hot += (double)wt[k];
      hot_seen = true;
      if (RULE == LV_RULE_CUDA_I && !(self_mask >> k & 1u)) own += (double)wt[k];
    }
    if (ins) {
      bool claimed;
      const uint32_t slot = table_claim(keys, mask, cu[k], L.sc, claimed);
      atomicAdd(&vals[slot], (double)wt[k]);
      if (claimed) claim_slot<MAXW>(slots, owned, k, slot);
    }
  }
}

template <int MODE>
__device__ __forceinline__ void block_body(const PassDesc* __restrict__ D, int cls, uint32_t bid,
                                           uint32_t nblk, unsigned char* smem_raw,
                                           typename BestOf<ModeOf<MODE>::kPrec>::T* red_best,
                                           double* red_own, const StepIO io = StepIO{}) {
  constexpr int RULE = ModeOf<MODE>::kRule, PREC = ModeOf<MODE>::kPrec;
  using K = typename BestOf<PREC>::T;
  const LevelView L = step_view(D, io);
  reapply_prev_step(D, io, bid, nblk);
  record_pass_start(D, L, io, bid, nblk);
  const uint32_t s0 = D->A.P.cls_start[cls];
  const uint32_t* __restrict__ verts = D->A.order + s0;
  uint32_t* __restrict__ prop = D->prop + s0;
  const uint32_t count = D->act_cnt ? D->act_cnt[cls] : D->A.P.cls_start[cls + 1] - s0;
  constexpr int T = kHubSmemSlots;
  constexpr int MAXW = (int)(kHubSmemMaxDeg / kThreads);
  double* vals = reinterpret_cast<double*>(smem_raw);
  uint32_t* keys = reinterpret_cast<uint32_t*>(smem_raw + sizeof(double) * T);
  uint32_t clean = 0;  // leading table slots known to be empty
  VertexRow nxt = fetch_vertex(L, verts, bid, count);
  for (uint32_t vidx = bid; vidx < count; vidx += nblk) {
    const uint32_t v = nxt.v;
    const uint64_t s = nxt.s;
    const uint32_t d = (uint32_t)(nxt.e - nxt.s);
    const uint32_t cv = nxt.cv;
    nxt = fetch_vertex(L, verts, vidx + nblk, count);
    if (!vertex_active(L, v)) {  // block-uniform: one vertex per block
      if (threadIdx.x == 0) prop[vidx] = cv;
      continue;
    }
    const uint32_t tv = table_size_for(d, T);
    if (tv > clean) {  // block-uniform; the scan empties what a row used
      for (uint32_t i = clean + threadIdx.x; i < tv; i += kThreads) {
        keys[i] = kEmptyKey;
        vals[i] = 0.0;
      }
      clean = tv;
      __syncthreads();
    }
    const GainCtx g = make_ctx<PREC>(L, v, cv);
    double own = 0.0;
    double hot = 0.0;
    bool hot_seen = false;
    uint32_t slots[(MAXW + 1) / 2] = {};
    uint32_t owned;
    insert_block_range<MAXW, RULE>(L, s, 0, d, v, cv, keys, vals, tv - 1, own, hot,
                                   hot_seen, slots, owned);
    // every warp adds its share of the own community's weight to that
    // community's slot (FP64 sums of FP32 weights are exact in any order),
    // so no block-wide sum is needed before the table is complete; the
    // warp whose add put the key in owns the candidate
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    hot = group_sum<32>(hot);
    uint32_t hot_slot = kEmptyKey;
    if (__any_sync(kFull, hot_seen) && lane == 0) {
      bool claimed;
      const uint32_t slot = table_claim(keys, tv - 1, cv, L.sc, claimed);
      atomicAdd(&vals[slot], hot);
      if (claimed) hot_slot = slot;
    }
    if (RULE == LV_RULE_CUDA_I) own = group_sum<32>(own);
    __syncthreads();  // (A) the table is complete
    K best = eval_owned<PREC, MAXW>(L, g, keys, vals, slots, owned, K{});
    if (hot_slot != kEmptyKey) best = eval_own_slot<PREC>(L, g, keys, vals, hot_slot, best);
    best = group_max<32>(best);
    if (lane == 0) {  // written after (A): thread 0 read the last ones before it
      red_best[wib] = best;
      if (RULE == LV_RULE_CUDA_I) red_own[wib] = own;
    }
    __syncthreads();  // (B) the table is empty again, the partials are in
    if (threadIdx.x == 0) {
      K b = red_best[0];
      double o = red_own[0];
      for (int i = 1; i < kWarps; i++) {
        b = best_max(b, red_best[i]);
        if (RULE == LV_RULE_CUDA_I) o += red_own[i];
      }
      record_decision(D, io, &prop[vidx], v, g,
                      decide<RULE>(b, RULE == LV_RULE_CUDA_I ? o : 0.0, g));
    }
    // no barrier here: the next vertex's first shared writes (the table's
    // inserts) touch no reduction slot, and the reduction slots are
    // rewritten only after the next (A), which thread 0 reaches after it
    // has read them
  }
}

// 319 < deg <= 2048: one block per vertex, shared 4096-slot table.
template <int MODE>
__global__ void __launch_bounds__(kThreads, kBlockPerSM)
    move_block_kernel(const PassDesc* __restrict__ D, int cls, StepIO io) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ typename BestOf<ModeOf<MODE>::kPrec>::T red_best[kWarps];
  __shared__ double red_own[kWarps];
  block_body<MODE>(D, cls, blockIdx.x, gridDim.x, smem_raw, red_best, red_own, io);
}

// deg > 2048 (hubs).  The neighbour communities of a hub are split into P
// hash partitions (P from the hub's degree, about kHubPartKeys distinct
// communities each).  hub_split_kernel: one block per kHubChunk-entry chunk
// of a hub row gathers the chunk's communities, sums the entries into the
// hub's own community on the spot and writes the others to the staging
// copy grouped by partition (a counting sort in shared memory), with the
// partition starts in the chunk table.  hub_merge_kernel: one block per
// (hub, partition) sums that partition's segments of all chunks in a
// self-cleaning shared table and folds its best candidate into the hub's
// packed (gain, ~community) key with one atomicMax.  Every hub entry is
// read once from the CSR and once from the staging copy; no global hash
// table, no per-entry global atomics.
__device__ __forceinline__ uint32_t hub_part_of(uint32_t c, uint32_t nparts) {
  return __umulhi(c * 0x85EBCA6Bu, nparts);
}

// In-place exclusive scan of a[0, n) (n <= kHubMaxParts) by the block;
// returns the total to every thread.
__device__ __forceinline__ uint32_t block_scan_inplace(uint32_t* a, uint32_t n,
                                                       uint32_t* wsum) {
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t per = (n + kThreads - 1) / kThreads;
  const uint32_t a0 = min(n, threadIdx.x * per), a1 = min(n, a0 + per);
  uint32_t local = 0;
  for (uint32_t i = a0; i < a1; i++) local += a[i];
  uint32_t incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[wib] = incl;
  __syncthreads();
  uint32_t before = 0, total = 0;
#pragma unroll
  for (int i = 0; i < kWarps; i++) {
    const uint32_t t = wsum[i];
    if (i < wib) before += t;
    total += t;
  }
  uint32_t run = before + incl - local;
  for (uint32_t i = a0; i < a1; i++) {
    const uint32_t t = a[i];
    a[i] = run;
    run += t;
  }
  __syncthreads();
  return total;
}

template <int MODE>
__device__ __forceinline__ void split_body(const PassDesc* __restrict__ D, uint32_t bid,
                                           uint32_t nblk, uint32_t* cnt, uint32_t* wsum,
                                           double* red, const StepIO io = StepIO{}) {
  constexpr int RULE = ModeOf<MODE>::kRule;
  const LevelView L = step_view(D, io);
  reapply_prev_step(D, io, bid, nblk);
  record_pass_start(D, L, io, bid, nblk);
  const uint32_t* __restrict__ hubs = D->A.order + D->A.P.cls_start[8];
  const HubArena H = D->H;
  const uint32_t nblocks = D->A.P.hub_blocks;
  const uint32_t* __restrict__ blk_hub = D->A.hub_blk_vertex;
  const uint32_t* __restrict__ blk_ch = D->A.hub_blk_chunk;
  constexpr int EPT = kHubChunk / kThreads;  // entries per thread
  static_assert(EPT * kThreads == (int)kHubChunk, "chunk = whole waves");
  for (uint32_t b = bid; b < nblocks; b += nblk) {
    const uint32_t hi = blk_hub[b], ch = blk_ch[b];
    const uint32_t v = hubs[hi];
    if (!vertex_active(L, v)) continue;  // block-uniform
    const uint64_t s = L.off[v];
    const uint64_t lo = (uint64_t)ch * kHubChunk;
    const uint64_t rest = L.off[v + 1] - s - lo;
    const uint32_t n_in = rest < kHubChunk ? (uint32_t)rest : kHubChunk;
    const uint32_t P = H.nparts[hi];
    const uint32_t cv = L.comm[v];
    for (uint32_t p = threadIdx.x; p < P; p += kThreads) cnt[p] = 0u;
    __syncthreads();
    uint32_t c[EPT], part[EPT], rank[EPT];
    float w[EPT];
    bool self[EPT];
#pragma unroll
    for (int k = 0; k < EPT; k++) {  // every load before any use
      const uint32_t j = k * kThreads + threadIdx.x;
      c[k] = v;
      w[k] = 0.0f;
      if (j < n_in) {
        c[k] = L.col[s + lo + j];
        w[k] = L.w[s + lo + j];
      }
    }
#pragma unroll
    for (int k = 0; k < EPT; k++) {
      const uint32_t j = k * kThreads + threadIdx.x;
      self[k] = c[k] == v;
      c[k] = (j < n_in) ? L.comm[c[k]] : kEmptyKey;
    }
    double hot = 0.0, own = 0.0;
    bool hot_seen = false;
#pragma unroll
    for (int k = 0; k < EPT; k++) {
      part[k] = kEmptyKey;
      if (c[k] == kEmptyKey) continue;
      if (c[k] == cv) {  // own community: summed here, not staged
        hot += (double)w[k];
        hot_seen = true;
        if (RULE == LV_RULE_CUDA_I && !self[k]) own += (double)w[k];
      } else {
        part[k] = hub_part_of(c[k], P);
        rank[k] = atomicAdd(&cnt[part[k]], 1u);
      }
    }
    __syncthreads();
    const uint32_t staged = block_scan_inplace(cnt, P, wsum);
    uint32_t* ct = H.ct + H.ct_off[hi] + (uint64_t)ch * (P + 1);
    for (uint32_t p = threadIdx.x; p < P; p += kThreads) ct[p] = cnt[p];
    if (threadIdx.x == 0) ct[P] = staged;
    const uint64_t base = H.stage_off[hi] + lo;
#pragma unroll
    for (int k = 0; k < EPT; k++) {
      if (part[k] == kEmptyKey) continue;
      const uint64_t pos = base + cnt[part[k]] + rank[k];
      H.stage[pos] = make_uint2(c[k], __float_as_uint(w[k]));
    }
    const int any_hot = __syncthreads_or(hot_seen);
    if (any_hot) {
      hot = block_sum(hot, red);
      if (threadIdx.x == 0) {
        atomicAdd(&H.hot[hi], hot);
        atomicOr(&H.hot_any[hi], 1u);
      }
    }
    if (RULE == LV_RULE_CUDA_I) {
      own = block_sum(own, red);
      if (threadIdx.x == 0 && own != 0.0) atomicAdd(&H.own[hi], own);
    }
    __syncthreads();  // cnt is reused by the next chunk
  }
}

template <int MODE>
__global__ void __launch_bounds__(kThreads, kSplitPerSM)
    hub_split_kernel(const PassDesc* __restrict__ D, StepIO io) {
  __shared__ uint32_t cnt[kHubMaxParts];
  __shared__ uint32_t wsum[kWarps];
  __shared__ double red[kWarps];
  split_body<MODE>(D, blockIdx.x, gridDim.x, cnt, wsum, red, io);
}

template <int MODE>
__device__ __forceinline__ void merge_body(const PassDesc* __restrict__ D, uint32_t bid,
                                           uint32_t nblk, unsigned char* smem_raw,
                                           typename BestOf<ModeOf<MODE>::kPrec>::T* red_best,
                                           uint32_t* seg_a, uint32_t* seg_pre, uint32_t* wsum,
                                           const StepIO io = StepIO{}) {
  constexpr int PREC = ModeOf<MODE>::kPrec;
  using K = typename BestOf<PREC>::T;
  const LevelView L = step_view(D, io);
  const uint32_t* __restrict__ hubs = D->A.order + D->A.P.cls_start[8];
  const HubArena H = D->H;
  const uint32_t units = H.units;
  constexpr int T = kHubPartSlots;
  double* vals = reinterpret_cast<double*>(smem_raw);
  uint32_t* keys = reinterpret_cast<uint32_t*>(smem_raw + sizeof(double) * T);
  for (uint32_t i = threadIdx.x; i < T; i += kThreads) {
    keys[i] = kEmptyKey;
    vals[i] = 0.0;
  }
  __syncthreads();
  for (uint32_t u = bid; u < units; u += nblk) {
    const uint32_t hi = H.blk_vertex[u], part = H.blk_chunk[u];
    const uint32_t P = H.blk_nchunks[u];
    const uint32_t v = hubs[hi];
    if (!vertex_active(L, v)) continue;  // block-uniform; decide keeps cv
    const uint64_t d = L.off[v + 1] - L.off[v];
    const uint32_t nch = (uint32_t)((d + kHubChunk - 1) / kHubChunk);
    const uint32_t* ct = H.ct + H.ct_off[hi];
    const uint64_t sb = H.stage_off[hi];
    // the partition's segments of up to kThreads chunks at a time, walked
    // as one flat range by the whole block
    for (uint32_t cb = 0; cb < nch; cb += kThreads) {
      const uint32_t nb = min((uint32_t)kThreads, nch - cb);
      uint32_t len = 0;
      if (threadIdx.x < nb) {
        const uint64_t r = (uint64_t)(cb + threadIdx.x) * (P + 1) + part;
        seg_a[threadIdx.x] = ct[r];
        len = ct[r + 1] - ct[r];
      }
      seg_pre[threadIdx.x] = len;
      __syncthreads();
      const uint32_t total = block_scan_inplace(seg_pre, kThreads, wsum);
      for (uint32_t f0 = 0; f0 < total; f0 += kThreads) {  // block-uniform
        const uint32_t f = f0 + threadIdx.x;
        const bool has = f < total;
        uint32_t c = 0;
        float w = 0.0f;
        if (has) {
          uint32_t lo = 0, hi2 = nb - 1;  // last segment starting at or before f
          while (lo < hi2) {
            const uint32_t mid = (lo + hi2 + 1) >> 1;
            if (seg_pre[mid] <= f) lo = mid; else hi2 = mid - 1;
          }
          const uint64_t pos = sb + (uint64_t)(cb + lo) * kHubChunk + seg_a[lo] + (f - seg_pre[lo]);
          const uint2 cw = H.stage[pos];
          c = cw.x;
          w = __uint_as_float(cw.y);
        }
        table_add_wave(keys, vals, T - 1, has, c, (double)w, L.sc);
      }
      __syncthreads();  // seg_a / seg_pre are refilled
    }
    const GainCtx g = make_ctx<PREC>(L, v, L.comm[v]);
    K best = scan_table_and_clear<PREC, true>(L, g, keys, vals, T, threadIdx.x, kThreads);
    best = block_max(best, red_best);
    if (threadIdx.x == 0) {
      if constexpr (PREC) {  // no 96-bit atomic: the decide kernel reduces the units
        H.unit_g[u] = best.g;
        H.unit_c[u] = best.c;
      } else if (best) {
        atomicMax(&H.best[hi], best);
      }
    }
    __syncthreads();
  }
}

template <int MODE>
__global__ void __launch_bounds__(kThreads, kMergePerSM)
    hub_merge_kernel(const PassDesc* __restrict__ D, StepIO io) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ typename BestOf<ModeOf<MODE>::kPrec>::T red_best[kWarps];
  __shared__ uint32_t seg_a[kThreads], seg_pre[kThreads], wsum[kWarps];
  merge_body<MODE>(D, blockIdx.x, gridDim.x, smem_raw, red_best, seg_a, seg_pre, wsum, io);
}

template <int MODE>
__device__ __forceinline__ void decide_body(const PassDesc* __restrict__ D, uint32_t bid,
                                            uint32_t nblk, const StepIO io = StepIO{}) {
  constexpr int RULE = ModeOf<MODE>::kRule, PREC = ModeOf<MODE>::kPrec;
  using K = typename BestOf<PREC>::T;
  const LevelView L = step_view(D, io);
  const uint32_t* __restrict__ hubs = D->A.order + D->A.P.cls_start[8];
  const HubArena H = D->H;
  const uint32_t hub_count = D->A.P.hub_count;
  uint32_t* __restrict__ prop = D->prop + D->A.P.cls_start[8];
  for (uint32_t i = bid * blockDim.x + threadIdx.x; i < hub_count; i += nblk * blockDim.x) {
    const uint32_t v = hubs[i];
    const GainCtx g = make_ctx<PREC>(L, v, L.comm[v]);
    K best{};
    if constexpr (PREC) {  // the hub's merge units, adjacent from unit_start[i]
      for (uint32_t u = H.unit_start[i]; u < H.unit_start[i + 1]; u++)
        best = best_max(best, Best64{H.unit_g[u], H.unit_c[u]});
    } else {
      best = H.best[i];
    }
    // the own community's candidate from the split pass's sums
    if (H.hot_any[i]) best = best_max(best, candidate<PREC>(L, g, g.cv, H.hot[i]));
    record_decision(D, io, &prop[i], v, g, decide<RULE>(best, H.own[i], g));
    H.best[i] = 0ull;
    H.own[i] = 0.0;
    H.hot[i] = 0.0;
    H.hot_any[i] = 0u;
  }
}

template <int MODE>
__global__ void hub_decide_kernel(const PassDesc* __restrict__ D, StepIO io) {
  decide_body<MODE>(D, blockIdx.x, gridDim.x, io);
}

// Applies a bucket's proposals (assignCommunity + incremental totals).
__device__ __forceinline__ void apply_body(const PassDesc* __restrict__ D, int lo_cls,
                                           int hi_cls, uint32_t bid, uint32_t nblk) {
  // classes lo..hi are adjacent in the lists (bucket 7 without compaction:
  // classes 7 and 8); with compaction a class's active prefix
  const LevelView L = D->L;
  const uint32_t s0 = D->A.P.cls_start[lo_cls];
  const uint32_t* __restrict__ verts = D->A.order + s0;
  // written by the move phase of the same persistent launch: a plain
  // (coherent) load, never the read-only path
  const uint32_t* prop = D->prop + s0;
  const uint32_t count = (D->act_cnt && lo_cls <= kMoveClasses)
                             ? D->act_cnt[lo_cls]
                             : D->A.P.cls_start[hi_cls + 1] - s0;
  for (uint32_t i = bid * kThreads + threadIdx.x; i < count; i += nblk * kThreads) {
    const uint32_t v = verts[i];
    const uint32_t nc = prop[i];
    const uint32_t oc = L.comm[v];
    if (nc != oc) {
      atomicSub(&L.comm_sz[oc], 1u);
      atomicAdd(&L.comm_sz[nc], 1u);
      const double kv = (double)L.k[v];
      atomicAdd(&L.tot[oc], -kv);
      atomicAdd(&L.tot[nc], kv);
      L.comm[v] = nc;
    }
  }
}

__global__ void __launch_bounds__(kThreads, kSweepPerSM)
    apply_kernel(const PassDesc* __restrict__ D, int lo_cls, int hi_cls) {
  apply_body(D, lo_cls, hi_cls, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------
// Class-dispatch row reductions (row sums at level start, modularity sweep)
// ---------------------------------------------------------------------------
// Row sum: k_v = (float) sum_j w_vj.  vertex() returns the vertex's share
// of its graph's accumulator (batched form).
struct RowSumOp {
  static constexpr GraphField kField = &GraphState::m_acc;
  static constexpr bool kAsq = false;
  __device__ bool row(const LevelView&, uint32_t) const { return true; }
  __device__ uint32_t ctx(const LevelView&, uint32_t) const { return 0; }
  __device__ double edge(const LevelView&, uint32_t, uint32_t, float w) const {
    return (double)w;
  }
  __device__ double vertex(const LevelView& L, uint32_t v, double sum,
                           double& part) const {
    const float kf = (float)sum;
    L.k[v] = kf;
    L.tot[v] = (double)kf;
    if (L.tot_alt) L.tot_alt[v] = (double)kf;
    part += (double)kf;
    return (double)kf;
  }
  __device__ void hub(const LevelView&, const DispatchArgs& A, uint32_t hi, uint32_t,
                      double sum, double&) const {
    atomicAdd(&A.hub_acc[hi], sum);
  }
};

// Intra-community weight: sum_j w_vj [comm(u) == comm(v)].
struct IntraOp {
  static constexpr GraphField kField = &GraphState::intra_acc;
  // batched form: the vertex's community total squared (community ids are
  // vertex ids), so an active graph's sum of a_c^2 comes with its rows
  static constexpr bool kAsq = true;
  __device__ bool row(const LevelView&, uint32_t) const { return true; }
  __device__ uint32_t ctx(const LevelView& L, uint32_t v) const {
    return L.comm[v];
  }
  __device__ double edge(const LevelView& L, uint32_t cv, uint32_t u,
                         float w) const {
    return L.comm[u] == cv ? (double)w : 0.0;
  }
  __device__ double vertex(const LevelView&, uint32_t, double sum, double& part) const {
    part += sum;
    return sum;
  }
  __device__ void hub(const LevelView& L, const DispatchArgs&, uint32_t, uint32_t v,
                      double sum, double& part) const {
    part += sum;
    if (L.gid && sum != 0.0) atomicAdd(&L.gs[L.gid[v]].intra_acc, sum);
  }
};

// Change of the intra-community weight over a pass (single graph): only the
// rows of vertices whose community at the pass's start (cs) differs from
// the current one are swept.  Entry (v, u) changes the sum by
// w ([c(u) == c(v)] - [cs(u) == cs(v)]); every edge is stored in both of
// its rows with the same weight, so an entry whose other end did not move
// (its row is not swept) counts for both copies.  FP64 sums of FP32
// weights are exact, so the updated sum equals a full sweep's.
struct DeltaIntraOp {
  const uint32_t* cs;
  static constexpr GraphField kField = &GraphState::intra_acc;
  static constexpr bool kAsq = false;
  __device__ bool row(const LevelView& L, uint32_t v) const { return cs[v] != L.comm[v]; }
  __device__ uint2 ctx(const LevelView& L, uint32_t v) const {
    return make_uint2(cs[v], L.comm[v]);
  }
  __device__ double edge(const LevelView& L, uint2 c, uint32_t u, float w) const {
    const uint32_t csu = cs[u], cu = L.comm[u];
    const bool was = csu == c.x, now = cu == c.y;
    if (was == now) return 0.0;
    const double x = (csu != cu) ? (double)w : 2.0 * (double)w;
    return now ? x : -x;
  }
  __device__ double vertex(const LevelView&, uint32_t, double sum, double& part) const {
    part += sum;
    return sum;
  }
  __device__ void hub(const LevelView&, const DispatchArgs&, uint32_t, uint32_t, double sum,
                      double& part) const {
    part += sum;
  }
};

__device__ __forceinline__ double sq(double a) { return a * a; }

// Length of class cls's list: the active length in the batched form's
// compacted lists, else the whole class.
__device__ __forceinline__ uint32_t class_count(const DispatchArgs& A, int cls) {
  return A.act_cnt ? A.act_cnt[cls] : A.P.cls_start[cls + 1] - A.P.cls_start[cls];
}

// Batched form, one lane for one vertex: its share of its graph's
// accumulator (and its community total squared for the sweep).
template <class Op>
__device__ __forceinline__ void graph_add_one(const LevelView& L, uint32_t v, double share) {
  GraphState& s = L.gs[L.gid[v]];
  if (share != 0.0) atomicAdd(&(s.*Op::kField), share);
  if (Op::kAsq) {
    const double a = L.tot[v];
    if (a != 0.0) atomicAdd(&s.asq_acc, a * a);
  }
}

template <int G, class Op>
__device__ __forceinline__ void unit_small(const LevelView& L,
                                           const DispatchArgs& A, int cls,
                                           uint32_t unit, const Op& op,
                                           double& part) {
  const int lane = threadIdx.x & 31, gl = lane & (G - 1);
  const uint32_t cnt = class_count(A, cls);
  const uint32_t idx = unit * (kThreads / G) + threadIdx.x / G;
  double x = 0.0;
  uint32_t v = 0;
  if (idx < cnt) {
    v = A.order[A.P.cls_start[cls] + idx];
    const uint64_t s = L.off[v];
    const uint32_t d = (uint32_t)(L.off[v + 1] - s);
    if (gl < (int)d && op.row(L, v)) {
      const auto c = op.ctx(L, v);
      x = op.edge(L, c, L.col[s + gl], L.w[s + gl]);
    }
  }
  x = group_sum<G>(x);
  double share = 0.0, a2 = 0.0;
  if (idx < cnt && gl == 0) {
    share = op.vertex(L, v, x, part);
    if (Op::kAsq && L.gid) a2 = sq(L.tot[v]);
  }
  if (L.gid) {  // warp-uniform
    const uint32_t key = idx < cnt ? L.gid[v] : kNoGraph;
    warp_graph_add(L.gs, Op::kField, key, share);
    if (Op::kAsq) warp_graph_add(L.gs, &GraphState::asq_acc, key, a2);
  }
}

template <class Op>
__device__ __forceinline__ void unit_warp(const LevelView& L,
                                          const DispatchArgs& A, int cls,
                                          uint32_t unit, const Op& op,
                                          double& part) {
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t cnt = class_count(A, cls);
  const uint32_t idx = unit * kWarps + wib;
  if (idx >= cnt) return;  // warp-uniform
  const uint32_t v = A.order[A.P.cls_start[cls] + idx];
  if (!op.row(L, v)) return;  // warp-uniform
  const uint64_t s = L.off[v];
  const uint32_t d = (uint32_t)(L.off[v + 1] - s);
  const auto c = op.ctx(L, v);
  double x = 0.0;
  for (uint32_t j = lane; j < d; j += 32) x += op.edge(L, c, L.col[s + j], L.w[s + j]);
  x = group_sum<32>(x);
  if (lane == 0) {
    const double share = op.vertex(L, v, x, part);
    if (L.gid) graph_add_one<Op>(L, v, share);
  }
}

template <class Op>
__device__ __forceinline__ void unit_block(const LevelView& L,
                                           const DispatchArgs& A,
                                           uint32_t unit, const Op& op,
                                           double& part, double* red) {
  const uint32_t idx = unit;
  if (idx >= class_count(A, 7)) return;  // block-uniform
  const uint32_t v = A.order[A.P.cls_start[7] + idx];
  if (!op.row(L, v)) return;  // block-uniform
  const uint64_t s = L.off[v];
  const uint32_t d = (uint32_t)(L.off[v + 1] - s);
  const auto c = op.ctx(L, v);
  double x = 0.0;
  for (uint32_t j = threadIdx.x; j < d; j += kThreads)
    x += op.edge(L, c, L.col[s + j], L.w[s + j]);
  x = block_sum(x, red);
  if (threadIdx.x == 0) {
    const double share = op.vertex(L, v, x, part);
    if (L.gid) graph_add_one<Op>(L, v, share);
  }
}

template <class Op>
__device__ __forceinline__ void unit_hub(const LevelView& L,
                                         const DispatchArgs& A, uint32_t unit,
                                         const Op& op, double& part,
                                         double* red) {
  const uint32_t hb = unit;
  const uint32_t hi = A.hub_blk_vertex[hb], ch = A.hub_blk_chunk[hb];
  const uint32_t v = A.order[A.P.cls_start[8] + hi];
  // batched pass loop: a finished graph's hubs need no sweep (block-uniform)
  if (A.act_cnt && !L.gs[L.gid[v]].active) return;
  if (!op.row(L, v)) return;  // block-uniform
  const uint64_t s = L.off[v];
  const uint64_t d = L.off[v + 1] - s;
  const uint64_t lo = (uint64_t)ch * kHubChunk, end = min(d, lo + kHubChunk);
  const auto c = op.ctx(L, v);
  double x = 0.0;
  for (uint64_t j = lo + threadIdx.x; j < end; j += kThreads)
    x += op.edge(L, c, L.col[s + j], L.w[s + j]);
  x = block_sum(x, red);
  if (threadIdx.x == 0) {
    op.hub(L, A, hi, v, x, part);
    if (Op::kAsq && L.gid && ch == 0 && L.tot[v] != 0.0)
      atomicAdd(&L.gs[L.gid[v]].asq_acc, sq(L.tot[v]));
  }
}

// Deterministic block reduction into partials, then the last block to
// finish sums all partials in index order.
__device__ __forceinline__ bool publish_and_check_last(double a, double b,
                                                       const DispatchArgs& A,
                                                       LevelScalars* sc,
                                                       double* red) {
  __shared__ bool last;
  double ra = block_sum(a, red);
  double rb = block_sum(b, red);
  if (threadIdx.x == 0) {
    A.partials[blockIdx.x] = ra;
    A.partials[gridDim.x + blockIdx.x] = rb;
    __threadfence();
    const uint32_t t = atomicAdd(&sc->done_blocks, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (last) __threadfence();
  return last;
}

__device__ __forceinline__ void sum_partials(const DispatchArgs& A, double* red,
                                             double& a, double& b) {
  double x = 0.0, y = 0.0;
  for (uint32_t i = threadIdx.x; i < gridDim.x; i += kThreads) {
    x += __ldcg(&A.partials[i]);
    y += __ldcg(&A.partials[gridDim.x + i]);
  }
  a = block_sum(x, red);
  b = block_sum(y, red);
}

// Units of the class lists, grid-strided.  Every unit function gets its
// unit's index within the class.  With act_cnt (batched pass loop) the
// classes 1..7 hold only their active prefix, so the unit ranges are
// derived from the device-side lengths and finished graphs cost nothing.
template <class Op>
__device__ __forceinline__ void dispatch_units(const LevelView& L,
                                               const DispatchArgs& A,
                                               const Op& op, double& part,
                                               double* red) {
  __shared__ uint32_t bs[kClasses + 1];
  if (threadIdx.x == 0) {
    if (A.act_cnt) {
      bs[0] = bs[1] = 0u;
      for (int c = 1; c <= kMoveClasses; c++) {
        const uint32_t pu = class_per_unit(c);
        bs[c + 1] = bs[c] + (A.act_cnt[c] + pu - 1) / pu;
      }
      bs[9] = bs[8] + A.P.hub_blocks;
    } else {
      for (int c = 0; c <= kClasses; c++) bs[c] = A.P.blk_start[c];
    }
  }
  __syncthreads();
  const uint32_t total = bs[9];
  for (uint32_t unit = blockIdx.x; unit < total; unit += gridDim.x) {
    int cls = 8;
    while (cls > 1 && unit < bs[cls]) cls--;
    const uint32_t u = unit - bs[cls];
    switch (cls) {  // block-uniform
      case 1: unit_small<4>(L, A, 1, u, op, part); break;
      case 2: unit_small<8>(L, A, 2, u, op, part); break;
      case 3: unit_small<16>(L, A, 3, u, op, part); break;
      case 4: unit_small<32>(L, A, 4, u, op, part); break;
      case 5:
      case 6: unit_warp(L, A, cls, u, op, part); break;
      case 7: unit_block(L, A, u, op, part, red); break;
      default: unit_hub(L, A, u, op, part, red); break;
    }
  }
}

__global__ void __launch_bounds__(kThreads)
    level_init_kernel(LevelView L, DispatchArgs A, uint32_t* __restrict__ rowid,
                      uint32_t* __restrict__ comm_start) {
  __shared__ double red[kWarps];
  double part = 0.0;
  dispatch_units(L, A, RowSumOp{}, part, red);
  // singleton state (modularity.cu:459-462), and for a single graph the
  // pass-start communities of the incremental sweep and the row of every
  // entry (the pass loop's flat modularity sweep).  A warp takes 32
  // consecutive ids, a lane each id's state and bounds, then writes the 32
  // rows' entry rows one row after another, 32 entries per store.
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t step = (uint64_t)gridDim.x * kWarps * 32;
  for (uint64_t v0 = ((uint64_t)blockIdx.x * kWarps + (threadIdx.x >> 5)) * 32; v0 < L.n;
       v0 += step) {  // warp-uniform
    const uint64_t c = v0 + lane;
    uint64_t s = 0, e = 0;
    if (c < L.n) {
      s = L.off[c];
      e = L.off[c + 1];
      L.comm[c] = (uint32_t)c;
      L.comm_sz[c] = 1u;
      if (L.comm_alt) {  // both copies of the state start equal
        L.comm_alt[c] = (uint32_t)c;
        L.sz_alt[c] = 1u;
      }
      if (comm_start) comm_start[c] = (uint32_t)c;
      if (e == s) {
        L.k[c] = 0.0f;
        L.tot[c] = 0.0;
        if (L.tot_alt) L.tot_alt[c] = 0.0;
      }
    }
    if (rowid) {
      for (int i = 0; i < 32; i++) {
        const uint64_t si = __shfl_sync(kFull, s, i), ei = __shfl_sync(kFull, e, i);
        for (uint64_t j = si + lane; j < ei; j += 32) rowid[j] = (uint32_t)(v0 + i);
      }
    }
  }
  if (!publish_and_check_last(part, 0.0, A, L.sc, red)) return;
  double msum, unused;
  sum_partials(A, red, msum, unused);
  // hubs: finalise their row sums in index order
  double hs = 0.0;
  for (uint32_t i = threadIdx.x; i < A.P.hub_count; i += kThreads) {
    const uint32_t v = A.order[A.P.cls_start[8] + i];
    const float kf = (float)__ldcg(&A.hub_acc[i]);
    L.k[v] = kf;
    L.tot[v] = (double)kf;
    if (L.tot_alt) L.tot_alt[v] = (double)kf;
    A.hub_acc[i] = 0.0;
    hs += (double)kf;
    if (L.gid && kf != 0.0f) atomicAdd(&L.gs[L.gid[v]].m_acc, (double)kf);
  }
  hs = block_sum(hs, red);
  if (threadIdx.x == 0) {
    const double m64 = (msum + hs) / 2.0;
    const float m = (float)m64;
    L.sc->m64 = m64;
    L.sc->m = m;
    L.sc->den = __fmul_rn(__fmul_rn(2.0f, m), m);
    L.sc->done_blocks = 0u;
  }
  // batched form: every graph's own m (the union's m above is unused)
  if (L.gid) {
    for (uint32_t g = threadIdx.x; g < L.n_graphs; g += kThreads) {
      GraphState& gs = L.gs[g];
      const double m64 = __ldcg(&gs.m_acc) / 2.0;
      const float m = (float)m64;
      gs.m64 = m64;
      gs.m = m;
      gs.den = __fmul_rn(__fmul_rn(2.0f, m), m);
      gs.m_acc = 0.0;
    }
  }
}

// Single graph with row ids: the intra-community weight over the entries
// themselves -- every load coalesced but the two community gathers, four
// independent entries per thread in flight.
__device__ __forceinline__ double intra_sweep(const LevelView& L, const uint32_t* rowid,
                                             uint64_t nnz, uint32_t bid, uint32_t nblk) {
  double part = 0.0;
  // 128-bit loads: a 4-entry vector of row ids, columns and weights per
  // thread and iteration (every array 16-byte aligned: the engine's own
  // buffers always are; a caller's may not be, and then the 32-bit loop
  // below takes every entry)
  uint64_t vec_end = 0;
  if ((((uintptr_t)rowid | (uintptr_t)L.col | (uintptr_t)L.w) & 15u) == 0) {
    const uint64_t nvec = nnz / 4;
    const uint4* __restrict__ r4 = reinterpret_cast<const uint4*>(rowid);
    const uint4* __restrict__ c4 = reinterpret_cast<const uint4*>(L.col);
    const float4* __restrict__ w4 = reinterpret_cast<const float4*>(L.w);
    const uint64_t vstride = (uint64_t)nblk * kThreads;
    for (uint64_t q = (uint64_t)bid * kThreads + threadIdx.x; q < nvec; q += vstride) {
      const uint4 r = __ldg(r4 + q);
      const uint4 c = __ldg(c4 + q);
      const float4 w = __ldg(w4 + q);
      const uint32_t a0 = L.comm[r.x], b0 = L.comm[c.x];
      const uint32_t a1 = L.comm[r.y], b1 = L.comm[c.y];
      const uint32_t a2 = L.comm[r.z], b2 = L.comm[c.z];
      const uint32_t a3 = L.comm[r.w], b3 = L.comm[c.w];
      if (a0 == b0) part += (double)w.x;
      if (a1 == b1) part += (double)w.y;
      if (a2 == b2) part += (double)w.z;
      if (a3 == b3) part += (double)w.w;
    }
    vec_end = nvec * 4;
  }
  // the entries after the last whole vector (or every entry, unaligned)
  const uint64_t stride = (uint64_t)nblk * kThreads * 4;
  for (uint64_t b = vec_end + (uint64_t)bid * kThreads * 4 + threadIdx.x; b < nnz; b += stride) {
    uint32_t r[4], c[4];
    float w[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const uint64_t j = b + (uint64_t)k * kThreads;
      r[k] = c[k] = 0u;
      w[k] = 0.0f;
      if (j < nnz) {
        r[k] = rowid[j];
        c[k] = L.col[j];
        w[k] = L.w[j];
      }
    }
#pragma unroll
    for (int k = 0; k < 4; k++)
      if (L.comm[r[k]] == L.comm[c[k]]) part += (double)w[k];
  }
  return part;
}

// Modularity of the current partition (modularity.cu:400-436): the
// intra-community weight (over the entries with row ids, else over the
// class lists) and the sum of squared community totals.
// cs (single graph, pass sweeps): every vertex's community when the pass
// began.  With it the sweep also counts the entries of the vertices that
// moved, and when the previous pass moved fewer than a quarter of the
// entries it updates the previous intra-community weight from the moved
// rows only (DeltaIntraOp) instead of sweeping every entry.
__device__ __forceinline__ void modularity_body(const LevelView& L, const DispatchArgs& A,
                                                const PassControl& ctl,
                                                const uint32_t* rowid, uint64_t nnz,
                                                const uint32_t* cs = nullptr) {
  __shared__ double red[kWarps];
  double part = 0.0;
  // read before this block publishes: the last block rewrites it
  const bool inc = cs && !L.gid && *(volatile uint32_t*)&L.sc->inc_next != 0u;
  if (inc) {
    dispatch_units(L, A, DeltaIntraOp{cs}, part, red);
  } else if (rowid && !L.gid) {
    part = intra_sweep(L, rowid, nnz, blockIdx.x, gridDim.x);
  } else {
    dispatch_units(L, A, IntraOp{}, part, red);
  }
  const uint32_t chunk = (L.n + gridDim.x - 1) / gridDim.x;
  const uint32_t c0 = blockIdx.x * chunk;
  const uint32_t c1 = min(L.n, c0 + chunk);
  double asq = 0.0;
  unsigned long long moved = 0ull;
  if (!L.gid) {  // the batched form summed a_c^2 with the rows above
    for (uint32_t c = c0 + threadIdx.x; c < c1; c += kThreads) {
      const double a = L.tot[c];
      asq += a * a;
      if (cs && cs[c] != L.comm[c]) moved += L.off[c + 1] - L.off[c];
    }
  }
  if (cs) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) moved += __shfl_xor_sync(kFull, moved, o);
    if ((threadIdx.x & 31) == 0 && moved) atomicAdd(&L.sc->moved_acc, moved);
  }
  if (!publish_and_check_last(part, asq, A, L.sc, red)) return;
  double intra, sq;
  sum_partials(A, red, intra, sq);
  if (!L.gid) {
    if (threadIdx.x == 0) {
      if (inc) intra += L.sc->intra;  // the pass's change added to the last sweep's sum
      const unsigned long long mv = cs ? atomicExch(&L.sc->moved_acc, 0ull) : 0ull;
      L.sc->inc_next = (cs && mv * 4ull < nnz) ? 1u : 0u;
      const double m = L.sc->m64;
      const double q = (m > 0.0) ? (intra / (2.0 * m)) - (sq / (4.0 * m * m)) : 0.0;
      L.sc->intra = intra;
      L.sc->asq = sq;
      L.sc->q = q;
      L.sc->done_blocks = 0u;
      if (ctl.enabled) {
        // stop rule of modularity.cu:501-508 / louvian.py:91-99
        const uint32_t p = L.sc->passes + 1;
        const double old = L.sc->q_prev;
        if (p == 1 && q - old < ctl.min_gain) L.sc->first_fail = 1u;
        const bool cont = (q - old >= ctl.min_gain) && p < ctl.max_passes;
        L.sc->passes = p;
        L.sc->q_before = old;
        L.sc->q_prev = q;
        L.sc->any_active = cont ? 1u : 0u;
        if (ctl.use_handle)
          cudaGraphSetConditional((cudaGraphConditionalHandle)ctl.handle, cont ? 1u : 0u);
      }
    }
    return;
  }
  // batched form: every graph's modularity and stop rule; the loop goes on
  // while any graph still gains
  int any = 0, stopped = 0;
  for (uint32_t g = threadIdx.x; g < L.n_graphs; g += kThreads) {
    GraphState& s = L.gs[g];
    const double gi = __ldcg(&s.intra_acc), gq = __ldcg(&s.asq_acc);
    s.intra_acc = 0.0;
    s.asq_acc = 0.0;
    if (ctl.enabled && !s.active) continue;  // finished its pass loop
    const double m = s.m64;
    const double q = (m > 0.0) ? (gi / (2.0 * m)) - (gq / (4.0 * m * m)) : 0.0;
    s.q = q;
    if (ctl.enabled) {
      const uint32_t p = s.passes + 1;
      const double old = s.q_prev;
      if (p == 1 && q - old < ctl.min_gain) s.first_fail = 1u;
      const bool cont = (q - old >= ctl.min_gain) && p < ctl.max_passes;
      s.passes = p;
      s.q_before = old;
      s.q_prev = q;
      s.active = cont ? 1u : 0u;
      any |= cont ? 1 : 0;
      stopped |= cont ? 0 : 1;
    }
  }
  any = __syncthreads_or(any);
  stopped = __syncthreads_or(stopped);
  if (threadIdx.x == 0) {
    L.sc->done_blocks = 0u;
    if (ctl.enabled) {
      L.sc->any_active = any ? 1u : 0u;
      L.sc->act_changed = stopped ? 1u : 0u;
      if (ctl.use_handle)
        cudaGraphSetConditional((cudaGraphConditionalHandle)ctl.handle, any ? 1u : 0u);
    }
  }
}

__global__ void __launch_bounds__(kThreads)
    modularity_kernel(LevelView L, DispatchArgs A, PassControl ctl) {
  modularity_body(L, A, ctl, nullptr, 0);
}

// The modularity sweep of a pass (level and stop-rule limits from the
// descriptor).
__global__ void __launch_bounds__(kThreads, kModPerSM)
    modularity_pass_kernel(const PassDesc* __restrict__ D, PassControl ctl, StepIO io) {
  ctl.min_gain = D->min_gain;
  ctl.max_passes = D->max_passes;
  // reads the copy holding every move of the pass; the last step's moves
  // go into the other copy, which leaves both equal for the next pass
  const LevelView L = step_view(D, io);
  reapply_prev_step(D, io, blockIdx.x, gridDim.x);
  modularity_body(L, D->A, ctl, D->rowid, D->nnz, D->comm_start);
}

__global__ void pass_control_init_kernel(const PassDesc* __restrict__ D, PassControl ctl) {
  LevelScalars* sc = D->L.sc;
  GraphState* gs = D->L.gid ? D->L.gs : nullptr;
  const uint32_t n_graphs = D->L.gid ? D->n_graphs : 0u;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) {
    sc->passes = 0u;
    sc->first_fail = 0u;
    sc->q_prev = sc->q;
    sc->q_before = sc->q;
    sc->q_start = sc->q;
    sc->any_active = 1u;
    sc->moved_acc = 0ull;
    sc->inc_next = 0u;  // the first pass of a level sweeps every entry
    sc->act_changed = 1u;  // the first pass builds the active lists
    // single graph: a level without edge weight runs no pass (its gains
    // would divide by m = 0); the host reads m after the level
    if (ctl.use_handle && !D->L.gid)
      cudaGraphSetConditional((cudaGraphConditionalHandle)ctl.handle, sc->m64 > 0.0 ? 1u : 0u);
  }
  for (uint32_t g = t; g < n_graphs; g += gridDim.x * blockDim.x) {
    GraphState& s = gs[g];
    s.passes = 0u;
    s.first_fail = 0u;
    s.q_prev = s.q;
    s.q_before = s.q;
    // nothing moves in an edgeless graph, nor in one the host froze
    s.active = (s.m64 > 0.0 && !s.frozen) ? 1u : 0u;
  }
}

// ---------------------------------------------------------------------------
// Persistent level kernel: a single graph's whole pass loop in one launch.
// The reference runs every bucket step, community update and modularity
// reduction as separate launches with host round trips
// (modularity.cu:466-508); here they are phases of one cooperative kernel
// separated by grid-wide barriers, so a pass costs no launch at all.  The
// phases run the same bodies as the standalone kernels, on one shared-memory
// arena sized for the largest table (the G-lane sums and the hub split's
// partition counters alias it).
// ---------------------------------------------------------------------------
constexpr int kLoopPerSM = 4;
constexpr int kLoopSmem = kBlockTabSmem;
static_assert(kLoopSmem >= kWarps * 512 * kSlotBytes && kLoopSmem >= kHubPartSmem &&
                  kLoopSmem >= (int)(kHubMaxParts * sizeof(uint32_t)) &&
                  kLoopSmem >= (int)(kWarps * 32 * sizeof(double)),
              "every phase's shared memory fits the arena");
// A barrier wait longer than this is a fault (a phase of the largest graphs
// lasts milliseconds): the block sets the abort flag and the kernel ends.
constexpr unsigned long long kBarrierTimeoutNs = 4000000000ull;

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier (every block is co-resident: cooperative launch).
// `epoch` counts the barriers this block has passed, so barrier k completes
// when k * nblk arrivals have been counted.  Returns false when the kernel
// must end: this block's wait gave up (it sets the abort flag and the error)
// or another block's did.
__device__ __forceinline__ bool grid_barrier(LevelLoopState* S, uint32_t nblk,
                                             unsigned long long& epoch, uint32_t* err,
                                             int* ok_sm) {
  __syncthreads();
  epoch++;
  if (threadIdx.x == 0) {
    const unsigned long long target = epoch * nblk;
    __threadfence();  // this block's writes before its arrival
    atomicAdd(&S->arrived, 1ull);
    int ok = 1;
    const unsigned long long t0 = global_ns();
    while (ld_acquire_u64(&S->arrived) < target) {
      if (*(volatile uint32_t*)&S->abort) {
        ok = 0;
        break;
      }
      if (global_ns() - t0 > kBarrierTimeoutNs) {
        atomicExch(&S->abort, 1u);
        atomicExch(err, kErrBarrierTimeout);
        ok = 0;
        break;
      }
      __nanosleep(32);
    }
    __threadfence();
    *ok_sm = ok;
  }
  __syncthreads();
  return *ok_sm != 0;
}

// The phases are called, not inlined: each body gets the register budget
// to itself instead of sharing one allocation across the whole loop.
template <int G, int MODE>
__device__ __noinline__ void small_phase(const PassDesc* __restrict__ D, int cls, uint32_t bid,
                                         uint32_t nblk, unsigned char* smem, StepIO io) {
  small_body<G, MODE>(D, cls, bid, nblk, reinterpret_cast<double(*)[32]>(smem), io);
}
template <int T, int MAXW, int MODE>
__device__ __noinline__ void warp_phase(const PassDesc* __restrict__ D, int cls, uint32_t bid,
                                        uint32_t nblk, unsigned char* smem, StepIO io) {
  warp_body<T, MAXW, MODE>(D, cls, bid, nblk, smem, io);
}
template <int MODE>
__device__ __noinline__ void block_phase(const PassDesc* __restrict__ D, int cls, uint32_t bid,
                                         uint32_t nblk, unsigned char* smem,
                                         typename BestOf<ModeOf<MODE>::kPrec>::T* red_best,
                                         double* red_d, StepIO io) {
  block_body<MODE>(D, cls, bid, nblk, smem, red_best, red_d, io);
}
template <int MODE>
__device__ __noinline__ void split_phase(const PassDesc* __restrict__ D, uint32_t bid,
                                         uint32_t nblk, unsigned char* smem, uint32_t* wsum,
                                         double* red_d, StepIO io) {
  split_body<MODE>(D, bid, nblk, reinterpret_cast<uint32_t*>(smem), wsum, red_d, io);
}
template <int MODE>
__device__ __noinline__ void merge_phase(const PassDesc* __restrict__ D, uint32_t bid,
                                         uint32_t nblk, unsigned char* smem,
                                         typename BestOf<ModeOf<MODE>::kPrec>::T* red_best,
                                         uint32_t* seg_a, uint32_t* seg_pre, uint32_t* wsum,
                                         StepIO io) {
  merge_body<MODE>(D, bid, nblk, smem, red_best, seg_a, seg_pre, wsum, io);
}
template <int MODE>
__device__ __noinline__ void decide_phase(const PassDesc* __restrict__ D, uint32_t bid,
                                          uint32_t nblk, StepIO io) {
  decide_body<MODE>(D, bid, nblk, io);
}
__device__ __noinline__ void apply_phase(const PassDesc* __restrict__ D, int lo, int hi,
                                         uint32_t bid, uint32_t nblk) {
  apply_body(D, lo, hi, bid, nblk);
}
// This block's shares of the intra-community weight and of the squared
// community totals (modularity.cu:400-436), in partials[bid] and
// partials[nblk + bid].
__device__ __noinline__ void modularity_share_phase(const PassDesc* __restrict__ D, uint32_t bid,
                                                    uint32_t nblk, double* red_d, StepIO io) {
  // fused steps: the copy holding every move of the pass; the last step's
  // moves go into the other copy
  const LevelView L = step_view(D, io);
  reapply_prev_step(D, io, bid, nblk);
  double part = intra_sweep(L, D->rowid, D->nnz, bid, nblk);
  const uint32_t chunk = (L.n + nblk - 1) / nblk;
  const uint32_t c0 = bid * chunk, c1 = min(L.n, c0 + chunk);
  double asq = 0.0;
  for (uint32_t c = c0 + threadIdx.x; c < c1; c += kThreads) {
    const double a = L.tot[c];
    asq += a * a;
  }
  part = block_sum(part, red_d);
  asq = block_sum(asq, red_d);
  if (threadIdx.x == 0) {
    D->A.partials[bid] = part;
    D->A.partials[nblk + bid] = asq;
  }
}

template <int MODE>
__device__ __forceinline__ void run_variant(int kv, const PassDesc* __restrict__ D, int cls,
                                            uint32_t bid, uint32_t nblk, unsigned char* smem,
                                            typename BestOf<ModeOf<MODE>::kPrec>::T* red_best,
                                            double* red_d, StepIO io) {
  switch (kv) {
    case KV_SMALL4: small_phase<4, MODE>(D, cls, bid, nblk, smem, io); break;
    case KV_SMALL8: small_phase<8, MODE>(D, cls, bid, nblk, smem, io); break;
    case KV_SMALL16: small_phase<16, MODE>(D, cls, bid, nblk, smem, io); break;
    case KV_SMALL32: small_phase<32, MODE>(D, cls, bid, nblk, smem, io); break;
    case KV_WARP128: warp_phase<128, 3, MODE>(D, cls, bid, nblk, smem, io); break;
    case KV_WARP512: warp_phase<512, 10, MODE>(D, cls, bid, nblk, smem, io); break;
    default: block_phase<MODE>(D, cls, bid, nblk, smem, red_best, red_d, io); break;
  }
}

template <int MODE>
__global__ void __launch_bounds__(kThreads, kLoopPerSM)
    level_loop_kernel(const PassDesc* __restrict__ D) {
  using K = typename BestOf<ModeOf<MODE>::kPrec>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ K red_best[kWarps];
  __shared__ double red_d[kWarps];
  __shared__ uint32_t seg_a[kThreads], seg_pre[kThreads], wsum[kWarps];
  __shared__ int ok_sm;
  __shared__ double q_sm[3];
  const uint32_t bid = blockIdx.x, nblk = gridDim.x;
  LevelLoopState* S = D->loop;
  const LevelView L = D->L;
  LevelScalars* sc = L.sc;
  const DispatchArgs& A = D->A;
  const bool timer = S->timing && bid == 0 && threadIdx.x == 0;
  unsigned long long epoch = 0, t_prev = timer ? global_ns() : 0ull;
  // ends a phase: barrier, then (timing) the phase's device time as block 0
  // saw it -- from the previous barrier's exit to this one's
  auto phase_end = [&](int kind) -> bool {
    if (!grid_barrier(S, nblk, epoch, &sc->error, &ok_sm)) return false;
    if (timer) {
      const unsigned long long t = global_ns();
      S->phase_ns[kind] += t - t_prev;
      S->phase_cnt[kind] += 1ull;
      t_prev = t;
    }
    return true;
  };
  // pass control (modularity.cu:466-508); every block holds the same copy
  double q_prev = sc->q;
  uint32_t passes = 0, first_fail = 0;
  const double min_gain = D->min_gain;
  const uint32_t max_passes = D->max_passes;
  const bool hubs = A.P.hub_count > 0;
  // fused steps (StepIO): no apply phase and no barrier after it; step s
  // reads copy s % 2 of the community state, the sweep re-applies the last
  // step's moves
  const int fused = D->fused ? 1 : 0;
  for (;;) {
    StepIO io{fused, 0, 0, 0};
    int step = 0;
    for (int b = 1; b <= kBuckets; b++) {
      const bool has = A.P.cls_start[b + 1] > A.P.cls_start[b];
      const bool hb = b == kBuckets && hubs;
      if (!has && !hb) continue;  // uniform: the plan is the level's
      io.parity = fused ? (step & 1) : 0;
      if (has) {
        run_variant<MODE>(D->tune[b], D, b, bid, nblk, smem_raw, red_best, red_d, io);
        io.prev_lo = io.prev_hi = 0;  // re-applied by this phase
      }
      if (hb) {
        split_phase<MODE>(D, bid, nblk, smem_raw, wsum, red_d, io);
        io.prev_lo = io.prev_hi = 0;
        if (!phase_end(b - 1)) return;
        merge_phase<MODE>(D, bid, nblk, smem_raw, red_best, seg_a, seg_pre, wsum, io);
        if (!phase_end(7)) return;
        decide_phase<MODE>(D, bid, nblk, io);
        if (!phase_end(7)) return;
      } else if (!phase_end(b - 1)) {
        return;
      }
      if (fused) {
        io.prev_lo = b;
        io.prev_hi = hb ? 8 : b;
        step++;
      } else {
        apply_phase(D, b, hb ? 8 : b, bid, nblk);
        if (!phase_end(8)) return;
      }
    }
    io.parity = fused ? (step & 1) : 0;
    // modularity of the pass: this block's shares ...
    modularity_share_phase(D, bid, nblk, red_d, io);
    if (!phase_end(9)) return;
    // ... then every block sums all shares in the same fixed order, so all
    // blocks hold the same Q and take the same stop decision
    double x = 0.0, y = 0.0;
    for (uint32_t i = threadIdx.x; i < nblk; i += kThreads) {
      x += __ldcg(&A.partials[i]);
      y += __ldcg(&A.partials[nblk + i]);
    }
    x = block_sum(x, red_d);
    y = block_sum(y, red_d);
    if (threadIdx.x == 0) {
      const double m = sc->m64;
      q_sm[0] = (m > 0.0) ? (x / (2.0 * m)) - (y / (4.0 * m * m)) : 0.0;
      q_sm[1] = x;
      q_sm[2] = y;
    }
    __syncthreads();
    const double q = q_sm[0];
    // stop rule of modularity.cu:501-508 / louvian.py:91-99
    passes++;
    if (passes == 1 && q - q_prev < min_gain) first_fail = 1u;
    const bool cont = (q - q_prev >= min_gain) && passes < max_passes;
    if (bid == 0 && threadIdx.x == 0) {
      sc->q = q;
      sc->intra = q_sm[1];
      sc->asq = q_sm[2];
      sc->passes = passes;
      sc->first_fail = first_fail;
      sc->q_before = q_prev;
      sc->q_prev = q;
      sc->any_active = cont ? 1u : 0u;
    }
    q_prev = q;
    if (!cont) break;
  }
}

// ---------------------------------------------------------------------------
// Small helpers
// ---------------------------------------------------------------------------
__global__ void compose_kernel(uint32_t* a, size_t n, const uint32_t* map) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    a[i] = map[a[i]];
}
__global__ void gather_kernel(uint32_t* out, const uint32_t* in, size_t n,
                              const uint32_t* map) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = map[in[i]];
}
__global__ void graph_ids_kernel(const uint32_t* goff, uint32_t n_graphs, uint32_t n,
                                 uint32_t* gid) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = n_graphs - 1;  // largest g with goff[g] <= v
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (goff[mid] <= v) lo = mid; else hi = mid - 1;
    }
    gid[v] = lo;
  }
}
__global__ void finalize_graphs_kernel(const uint32_t* asg, size_t n0,
                                       const uint32_t* graph0, const uint32_t* base,
                                       uint32_t* out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n0;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t b = base[graph0[i]];
    if (b != 0xFFFFFFFFu) out[i] = asg[i] - b;
  }
}
__global__ void drop_graphs_kernel(uint32_t* comm_sz, const uint32_t* gid, uint32_t n,
                                   const uint32_t* drop) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += gridDim.x * blockDim.x)
    if (drop[gid[v]]) comm_sz[v] = 0u;
}
__global__ void gather_u32_kernel(const uint32_t* src, const uint32_t* idx, uint32_t n,
                                  uint32_t* out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x)
    out[i] = src[idx[i]];
}
__global__ void iota_kernel(uint32_t* a, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    a[i] = (uint32_t)i;
}
// Served form: arena and union-append helpers.
__global__ void iota_from_kernel(uint32_t* a, size_t n, uint32_t start) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    a[i] = start + (uint32_t)i;
}
__global__ void fill_u32_kernel(uint32_t* a, size_t n, uint32_t v) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    a[i] = v;
}
__global__ void add_u32_kernel(uint32_t* a, size_t n, uint32_t d) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    a[i] += d;
}
__global__ void add_u64_kernel(uint64_t* a, size_t n, uint64_t d) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    a[i] += d;
}
__global__ void recount_zero_kernel(LevelView L) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < L.n;
       i += gridDim.x * blockDim.x) {
    L.comm_sz[i] = 0u;
    L.tot[i] = 0.0;
  }
}
__global__ void recount_kernel(LevelView L) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < L.n;
       v += gridDim.x * blockDim.x) {
    const uint32_t c = L.comm[v];
    atomicAdd(&L.comm_sz[c], 1u);
    atomicAdd(&L.tot[c], (double)L.k[v]);
  }
}
__global__ void bucket_ids_kernel(const uint64_t* off, uint32_t n, uint8_t* out) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += gridDim.x * blockDim.x) {
    const uint64_t d = off[v + 1] - off[v];
    int c = move_class_of_degree(d);
    out[v] = (uint8_t)(c == 8 ? 7 : c);
  }
}
// FP64 modularity of an arbitrary partition (part[v] < n).
__global__ void part_totals_kernel(const LevelView L, const uint32_t* part,
                                   double* tot) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < L.n;
       v += gridDim.x * blockDim.x) {
    double k = 0.0;
    for (uint64_t j = L.off[v]; j < L.off[v + 1]; j++) k += (double)L.w[j];
    atomicAdd(&tot[part[v]], k);
  }
}
__global__ void part_q_kernel(const LevelView L, const uint32_t* part,
                              const double* tot, double* out /*[3]*/) {
  __shared__ double red[kWarps];
  double intra = 0.0, sq = 0.0, all = 0.0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < L.n;
       v += gridDim.x * blockDim.x) {
    const uint32_t p = part[v];
    for (uint64_t j = L.off[v]; j < L.off[v + 1]; j++) {
      all += (double)L.w[j];
      if (part[L.col[j]] == p) intra += (double)L.w[j];
    }
    sq += tot[v] * tot[v];
  }
  intra = block_sum(intra, red);
  sq = block_sum(sq, red);
  all = block_sum(all, red);
  if (threadIdx.x == 0) {
    atomicAdd(&out[0], intra);
    atomicAdd(&out[1], sq);
    atomicAdd(&out[2], all);
  }
}

unsigned grid_for(uint64_t work_blocks, unsigned cap) {
  if (work_blocks == 0) return 0;
  return (unsigned)(work_blocks < cap ? work_blocks : cap);
}

unsigned sm_count() { return sm_count_cached(); }

DispatchArgs make_args(const uint32_t* order, const DispatchPlan& P,
                       const uint32_t* hub_map, double* partials) {
  DispatchArgs A;
  A.P = P;
  A.order = order;
  A.hub_blk_vertex = hub_map;
  A.hub_blk_chunk = hub_map ? hub_map + P.hub_blocks : nullptr;
  A.hub_acc = partials;  // first hub_count doubles; partials follow
  A.partials = partials + P.hub_count;
  A.act_cnt = nullptr;
  return A;
}

}  // namespace

DispatchArgs dispatch_args(const uint32_t* order, const DispatchPlan& P, const uint32_t* hub_map,
                           double* partials) {
  return make_args(order, P, hub_map, partials);
}

unsigned sm_count_cached() {
  static int num_sms = 0;
  if (!num_sms) {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    num_sms = v > 0 ? v : 148;
  }
  return (unsigned)num_sms;
}

template <int MODE>
static cudaError_t configure_mode() {
  const int warp512 = kWarps * 512 * kSlotBytes;
  cudaError_t e = cudaFuncSetAttribute(move_warp_kernel<512, 10, MODE>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, warp512);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(move_block_kernel<MODE>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, kBlockTabSmem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(hub_merge_kernel<MODE>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, kHubPartSmem);
}

template <int MODE>
static cudaError_t configure_loop() {
  return cudaFuncSetAttribute(level_loop_kernel<MODE>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, kLoopSmem);
}

cudaError_t configure_kernels() {
  cudaError_t e;
  if ((e = configure_loop<0>()) != cudaSuccess) return e;
  if ((e = configure_loop<1>()) != cudaSuccess) return e;
  if ((e = configure_loop<2>()) != cudaSuccess) return e;
  if ((e = configure_loop<3>()) != cudaSuccess) return e;
  if ((e = configure_mode<0>()) != cudaSuccess) return e;
  if ((e = configure_mode<1>()) != cudaSuccess) return e;
  if ((e = configure_mode<2>()) != cudaSuccess) return e;
  if ((e = configure_mode<3>()) != cudaSuccess) return e;
  return configure_contract_kernels();
}

unsigned dispatch_grid(const DispatchPlan& P) {
  return grid_for(P.total_blocks ? P.total_blocks : 1, sm_count() * 8);
}

cudaError_t launch_level_init(const LevelView& L, const uint32_t* order,
                              const DispatchPlan& P, const uint32_t* hub_map,
                              double* partials, uint32_t* rowid, uint32_t* comm_start,
                              cudaStream_t st) {
  DispatchArgs A = make_args(order, P, hub_map, partials);
  (count_launches(1), level_init_kernel<<<dispatch_grid(P), kThreads, 0, st>>>(L, A, rowid,
                                                                             comm_start));
  return cudaGetLastError();
}

cudaError_t launch_modularity(const LevelView& L, const uint32_t* order,
                              const DispatchPlan& P, const uint32_t* hub_map,
                              double* partials, cudaStream_t st) {
  DispatchArgs A = make_args(order, P, hub_map, partials);
  PassControl c{};
  (count_launches(1), modularity_kernel<<<dispatch_grid(P), kThreads, 0, st>>>(L, A, c));
  return cudaGetLastError();
}

// Row of every entry.  A warp takes 32 consecutive rows: each lane loads
// one row's bounds, then the warp writes the 32 rows one after another,
// 32 entries per store (coalesced).  O(rows / 32 + entries / 32) steps per
// warp, whether the rows are long (hubs) or mostly empty (late levels).
__global__ void row_ids_kernel(const uint64_t* __restrict__ off, uint32_t n,
                               uint32_t* __restrict__ rowid) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t step = (uint64_t)gridDim.x * (blockDim.x / 32) * 32;
  for (uint64_t v0 = ((uint64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5)) * 32; v0 < n;
       v0 += step) {
    const uint64_t v = v0 + lane;
    uint64_t s = 0, e = 0;
    if (v < n) {
      s = off[v];
      e = off[v + 1];
    }
    for (int i = 0; i < 32; i++) {
      const uint64_t si = __shfl_sync(kFull, s, i), ei = __shfl_sync(kFull, e, i);
      for (uint64_t j = si + lane; j < ei; j += 32) rowid[j] = (uint32_t)(v0 + i);
    }
  }
}

// ---------------------------------------------------------------------------
// Pass kernels.  Every launch reads the level from the descriptor and uses
// a fixed grid (grid-stride loops end at the level's counts), so a pass
// captured once replays on any level.
// ---------------------------------------------------------------------------
cudaError_t launch_row_ids(const uint64_t* off, uint32_t n, uint64_t nnz, uint32_t* rowid,
                           cudaStream_t st) {
  if (nnz == 0 || n == 0) return cudaSuccess;
  const uint64_t groups = ((uint64_t)n + 31) / 32;  // a warp per 32 rows
  const unsigned grid = grid_for((groups + 7) / 8, sm_count() * 8);
  (count_launches(1), row_ids_kernel<<<grid, 256, 0, st>>>(off, n, rowid));
  return cudaGetLastError();
}

cudaError_t launch_pass_control_init(const PassDesc* D, const PassControl* ctl, cudaStream_t st) {
  PassControl c{};
  if (ctl) c = *ctl;
  (count_launches(1), pass_control_init_kernel<<<sm_count(), 256, 0, st>>>(D, c));
  return cudaGetLastError();
}

cudaError_t launch_modularity_pass(const PassDesc* D, const PassControl* ctl, cudaStream_t st,
                                   StepIO io) {
  PassControl c{};
  if (ctl) c = *ctl;
  (count_launches(1), modularity_pass_kernel<<<sm_count() * kModPerSM, kThreads, 0, st>>>(D, c, io));
  return cudaGetLastError();
}

unsigned pass_dispatch_grid() { return sm_count() * kModPerSM; }
unsigned move_block_resident() { return sm_count() * kBlockPerSM; }

// One launch of a move kernel variant over class `cls`.
template <int MODE>
static void launch_variant(int kv, const PassDesc* D, int cls, cudaStream_t st, StepIO io) {
  const unsigned cap = sm_count() * kSmallPerSM;
  switch (kv) {
    case KV_SMALL4:
      (count_launches(1), move_small_kernel<4, MODE><<<cap, kThreads, 0, st>>>(D, cls, io));
      break;
    case KV_SMALL8:
      (count_launches(1), move_small_kernel<8, MODE><<<cap, kThreads, 0, st>>>(D, cls, io));
      break;
    case KV_SMALL16:
      (count_launches(1), move_small_kernel<16, MODE><<<cap, kThreads, 0, st>>>(D, cls, io));
      break;
    case KV_SMALL32:
      (count_launches(1), move_small_kernel<32, MODE><<<cap, kThreads, 0, st>>>(D, cls, io));
      break;
    case KV_WARP128: {
      constexpr int T = 128;
      (count_launches(1), move_warp_kernel<T, 3, MODE><<<sm_count() * kWarp128PerSM, kThreads,
                                                       kWarps * T * kSlotBytes, st>>>(D, cls, io));
      break;
    }
    case KV_WARP512: {
      constexpr int T = 512;
      (count_launches(1), move_warp_kernel<T, 10, MODE><<<sm_count() * kWarp512PerSM, kThreads,
                                                        kWarps * T * kSlotBytes, st>>>(D, cls, io));
      break;
    }
    default:  // KV_BLOCK: shared table, one block per vertex
      (count_launches(1), move_block_kernel<MODE><<<sm_count() * kBlockPerSM, kThreads,
                                                   kBlockTabSmem, st>>>(D, cls, io));
      break;
  }
}

template <int MODE>
static cudaError_t move_bucket_impl(const PassDesc* D, int bucket, const uint8_t* kv,
                                    cudaStream_t st, StepIO io) {
  if (bucket >= 1 && bucket <= 7) {
    const int v = kv ? kv[bucket] : kDefaultVariant[bucket];
    if (!variant_fits(v, bucket)) return cudaErrorInvalidValue;
    launch_variant<MODE>(v, D, bucket, st, io);
    return cudaGetLastError();
  }
  if (bucket != 8) return cudaErrorInvalidValue;
  // class 8 of bucket 7: split chunks, merge (hub, partition), decide; the
  // split re-applies the previous step's moves, the decide kernel applies
  // the hubs' own
  StepIO later = io;
  later.prev_lo = later.prev_hi = 0;
  later.pass_start = 0;
  (count_launches(1), hub_split_kernel<MODE><<<sm_count() * kSplitPerSM, kThreads, 0, st>>>(D, io));
  (count_launches(1), hub_merge_kernel<MODE><<<sm_count() * kMergePerSM, kThreads, kHubPartSmem,
                                               st>>>(D, later));
  (count_launches(1), hub_decide_kernel<MODE><<<sm_count() * 2, 128, 0, st>>>(D, later));
  return cudaGetLastError();
}

cudaError_t launch_move_bucket(const PassDesc* D, int bucket, int mode, const uint8_t* variant,
                               cudaStream_t st, StepIO io) {
  switch (mode) {
    case 0: return move_bucket_impl<0>(D, bucket, variant, st, io);
    case 1: return move_bucket_impl<1>(D, bucket, variant, st, io);
    case 2: return move_bucket_impl<2>(D, bucket, variant, st, io);
    case 3: return move_bucket_impl<3>(D, bucket, variant, st, io);
    default: return cudaErrorInvalidValue;
  }
}

template <int MODE>
static unsigned loop_grid_impl() {
  static int per_sm = -1;  // co-resident blocks of the kernel, once per process
  if (per_sm < 0) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, level_loop_kernel<MODE>, kThreads,
                                                      kLoopSmem) != cudaSuccess)
      b = 0;
    per_sm = std::min(b, kLoopPerSM);
  }
  return (unsigned)per_sm * sm_count();
}

unsigned level_loop_grid(int mode) {
  switch (mode) {
    case 0: return loop_grid_impl<0>();
    case 1: return loop_grid_impl<1>();
    case 2: return loop_grid_impl<2>();
    case 3: return loop_grid_impl<3>();
    default: return 0;
  }
}

template <int MODE>
static cudaError_t launch_loop_impl(const PassDesc* D, cudaStream_t st) {
  const unsigned grid = loop_grid_impl<MODE>();
  if (!grid) return cudaErrorCooperativeLaunchTooLarge;
  void* args[] = {(void*)&D};
  count_launches(1);
  return cudaLaunchCooperativeKernel((const void*)level_loop_kernel<MODE>, dim3(grid),
                                     dim3(kThreads), args, kLoopSmem, st);
}

cudaError_t launch_level_loop(const PassDesc* D, int mode, cudaStream_t st) {
  switch (mode) {
    case 0: return launch_loop_impl<0>(D, st);
    case 1: return launch_loop_impl<1>(D, st);
    case 2: return launch_loop_impl<2>(D, st);
    case 3: return launch_loop_impl<3>(D, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_apply_bucket(const PassDesc* D, int bucket, bool compacted, cudaStream_t st) {
  const unsigned cap = sm_count() * kSweepPerSM;
  if (bucket == 7 && !compacted) {  // classes 7 and 8 are adjacent
    (count_launches(1), apply_kernel<<<cap, kThreads, 0, st>>>(D, 7, 8));
  } else if (bucket == 7) {  // class 7's active prefix, then the hubs
    (count_launches(1), apply_kernel<<<cap, kThreads, 0, st>>>(D, 7, 7));
    (count_launches(1), apply_kernel<<<cap, kThreads, 0, st>>>(D, 8, 8));
  } else {
    (count_launches(1), apply_kernel<<<cap, kThreads, 0, st>>>(D, bucket, bucket));
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Batched form: per-pass lists of the vertices whose graph still moves.
// A class list is ascending in vertex id and a graph owns a contiguous id
// range, so graph g's vertices form one run of every class list; the
// compacted list keeps the runs of active graphs in order.
// ---------------------------------------------------------------------------
__global__ void class_graph_starts_kernel(const uint32_t* __restrict__ order, ClassStarts cs,
                                          const uint32_t* __restrict__ goff, uint32_t G,
                                          uint32_t* __restrict__ cg) {
  const uint32_t per = G + 1;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < kMoveClasses * per;
       t += gridDim.x * blockDim.x) {
    const uint32_t c = 1 + t / per, g = t % per;
    const uint32_t* list = order + cs.s[c];
    const uint32_t n = cs.s[c + 1] - cs.s[c];
    const uint32_t key = goff[g];
    uint32_t lo = 0, hi = n;  // first index with list[i] >= key
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (list[mid] < key) lo = mid + 1; else hi = mid;
    }
    cg[t] = lo;
  }
}

// One block per class: exclusive scan over graphs of the active run
// lengths -> each active run's place in the compacted list, and the
// class's active count.  Skipped while the active set is unchanged.
__global__ void __launch_bounds__(1024)
    compact_scan_kernel(const PassDesc* __restrict__ D) {
  const uint32_t* __restrict__ cg = D->cg;
  const GraphState* __restrict__ gs = D->L.gs;
  const uint32_t G = D->n_graphs;
  uint32_t* __restrict__ cg_new = D->cg_new;
  uint32_t* __restrict__ act_cnt = D->act_cnt;
  if (!D->L.sc->act_changed) return;  // block-uniform
  __shared__ uint32_t warp_tot[32];
  __shared__ uint32_t carry;
  const uint32_t per = G + 1, c = blockIdx.x;
  const uint32_t* row = cg + c * per;
  uint32_t* out = cg_new + c * per;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0u;
  __syncthreads();
  for (uint32_t b = 0; b < G; b += 1024) {
    const uint32_t g = b + threadIdx.x;
    const uint32_t len = (g < G && gs[g].active) ? row[g + 1] - row[g] : 0u;
    uint32_t x = len;  // inclusive warp scan
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    if (wid == 0) {
      uint32_t t = warp_tot[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, t, o);
        if (lane >= o) t += y;
      }
      warp_tot[lane] = t;  // inclusive over warps
    }
    __syncthreads();
    const uint32_t before = carry + (wid ? warp_tot[wid - 1] : 0u) + x - len;
    if (g < G) out[g] = before;
    __syncthreads();
    if (threadIdx.x == 1023) carry = before + len;
    __syncthreads();
  }
  if (threadIdx.x == 0) act_cnt[1 + c] = carry;
}

// Fills the compacted lists: one thread per output position (blockIdx.y =
// class), its graph found by binary search over the runs' new starts (an
// inactive graph's empty run shares its start with the next graph, and the
// search takes the last of equal starts).  Skipped while the active set is
// unchanged.
__global__ void compact_copy_kernel(const PassDesc* __restrict__ D) {
  if (!D->L.sc->act_changed) return;
  const uint32_t* __restrict__ order = D->full_order;
  uint32_t* __restrict__ act_order = D->act_order;
  const uint32_t G = D->n_graphs;
  const uint32_t ci = blockIdx.y, per = G + 1;
  const uint32_t total = D->act_cnt[1 + ci];
  const uint32_t* row = D->cg + ci * per;
  const uint32_t* row_new = D->cg_new + ci * per;
  const uint32_t base = D->A.P.cls_start[ci + 1];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = G - 1;  // last g with row_new[g] <= i
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (row_new[mid] <= i) lo = mid; else hi = mid - 1;
    }
    act_order[base + i] = order[base + row[lo] + (i - row_new[lo])];
  }
}

cudaError_t launch_class_graph_starts(const uint32_t* order, const DispatchPlan& P,
                                      const uint32_t* goff, uint32_t G, uint32_t* cg,
                                      cudaStream_t st) {
  ClassStarts cs;
  for (int c = 0; c <= kClasses; c++) cs.s[c] = P.cls_start[c];
  if (!G) return cudaSuccess;
  const uint32_t total = kMoveClasses * (G + 1);
  (count_launches(1), class_graph_starts_kernel<<<grid_for((total + 255) / 256, sm_count() * 8), 256, 0, st>>>(
      order, cs, goff, G, cg));
  return cudaGetLastError();
}

cudaError_t launch_compact_active(const PassDesc* D, cudaStream_t st) {
  (count_launches(1), compact_scan_kernel<<<kMoveClasses, 1024, 0, st>>>(D));
  const dim3 grid(sm_count() * 2, kMoveClasses);
  (count_launches(1), compact_copy_kernel<<<grid, 256, 0, st>>>(D));
  return cudaGetLastError();
}

cudaError_t launch_compose(uint32_t* assignment, size_t n0,
                           const uint32_t* map, cudaStream_t st) {
  if (!n0) return cudaSuccess;
  (count_launches(1), compose_kernel<<<grid_for((n0 + 255) / 256, sm_count() * 8), 256, 0, st>>>(assignment, n0, map));
  return cudaGetLastError();
}

cudaError_t launch_gather(uint32_t* out, const uint32_t* in, size_t n,
                          const uint32_t* map, cudaStream_t st) {
  if (!n) return cudaSuccess;
  (count_launches(1), gather_kernel<<<grid_for((n + 255) / 256, sm_count() * 8), 256, 0, st>>>(
      out, in, n, map));
  return cudaGetLastError();
}

cudaError_t launch_graph_ids(const uint32_t* goff, uint32_t n_graphs, uint32_t n,
                             uint32_t* gid, cudaStream_t st) {
  if (!n || !n_graphs) return cudaSuccess;
  (count_launches(1), graph_ids_kernel<<<grid_for((n + 255) / 256, sm_count() * 8), 256, 0, st>>>(
      goff, n_graphs, n, gid));
  return cudaGetLastError();
}

cudaError_t launch_finalize_graphs(const uint32_t* asg, size_t n0, const uint32_t* graph0,
                                   const uint32_t* base, uint32_t* out, cudaStream_t st) {
  if (!n0) return cudaSuccess;
  (count_launches(1), finalize_graphs_kernel<<<grid_for((n0 + 255) / 256, sm_count() * 8), 256, 0, st>>>(
      asg, n0, graph0, base, out));
  return cudaGetLastError();
}

cudaError_t launch_drop_graphs(uint32_t* comm_sz, const uint32_t* gid, uint32_t n,
                               const uint32_t* drop, cudaStream_t st) {
  if (!n) return cudaSuccess;
  (count_launches(1), drop_graphs_kernel<<<grid_for((n + 255) / 256, sm_count() * 8), 256, 0, st>>>(
      comm_sz, gid, n, drop));
  return cudaGetLastError();
}

cudaError_t launch_gather_u32(const uint32_t* src, const uint32_t* idx, uint32_t n,
                              uint32_t* out, cudaStream_t st) {
  if (!n) return cudaSuccess;
  (count_launches(1), gather_u32_kernel<<<grid_for((n + 255) / 256, sm_count() * 8), 256, 0, st>>>(
      src, idx, n, out));
  return cudaGetLastError();
}

cudaError_t launch_iota_from(uint32_t* a, size_t n, uint32_t start, cudaStream_t st) {
  if (!n) return cudaSuccess;
  (count_launches(1), iota_from_kernel<<<grid_for((n + 255) / 256, sm_count() * 8), 256, 0, st>>>(
      a, n, start));
  return cudaGetLastError();
}
cudaError_t launch_fill_u32(uint32_t* a, size_t n, uint32_t v, cudaStream_t st) {
  if (!n) return cudaSuccess;
  (count_launches(1), fill_u32_kernel<<<grid_for((n + 255) / 256, sm_count() * 8), 256, 0, st>>>(
      a, n, v));
  return cudaGetLastError();
}
cudaError_t launch_add_u32(uint32_t* a, size_t n, uint32_t d, cudaStream_t st) {
  if (!n) return cudaSuccess;
  (count_launches(1), add_u32_kernel<<<grid_for((n + 255) / 256, sm_count() * 8), 256, 0, st>>>(
      a, n, d));
  return cudaGetLastError();
}
cudaError_t launch_add_u64(uint64_t* a, size_t n, uint64_t d, cudaStream_t st) {
  if (!n) return cudaSuccess;
  (count_launches(1), add_u64_kernel<<<grid_for((n + 255) / 256, sm_count() * 8), 256, 0, st>>>(
      a, n, d));
  return cudaGetLastError();
}

cudaError_t launch_fill_iota(uint32_t* a, size_t n, cudaStream_t st) {
  if (!n) return cudaSuccess;
  (count_launches(1), iota_kernel<<<grid_for((n + 255) / 256, sm_count() * 8), 256, 0, st>>>(a, n));
  return cudaGetLastError();
}

cudaError_t launch_recount(const LevelView& L, cudaStream_t st) {
  if (!L.n) return cudaSuccess;
  const unsigned g = grid_for((L.n + 255) / 256, sm_count() * 8);
  (count_launches(1), recount_zero_kernel<<<g, 256, 0, st>>>(L));
  (count_launches(1), recount_kernel<<<g, 256, 0, st>>>(L));
  return cudaGetLastError();
}

cudaError_t launch_bucket_ids(const uint64_t* off, uint32_t n, uint8_t* out,
                              cudaStream_t st) {
  if (!n) return cudaSuccess;
  (count_launches(1), bucket_ids_kernel<<<grid_for((n + 255) / 256, sm_count() * 8), 256, 0, st>>>(off, n, out));
  return cudaGetLastError();
}

cudaError_t launch_modularity_of(const LevelView& L, const uint32_t* part,
                                 double* tot_scratch, double* out,
                                 cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(tot_scratch, 0, sizeof(double) * (L.n ? L.n : 1), st);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(out, 0, sizeof(double) * 3, st);
  if (e != cudaSuccess) return e;
  if (!L.n) return cudaSuccess;
  const unsigned g = grid_for((L.n + 255) / 256, sm_count() * 8);
  (count_launches(1), part_totals_kernel<<<g, 256, 0, st>>>(L, part, tot_scratch));
  (count_launches(1), part_q_kernel<<<g, kThreads, 0, st>>>(L, part, tot_scratch, out));
  return cudaGetLastError();
}

}  // namespace lvb
