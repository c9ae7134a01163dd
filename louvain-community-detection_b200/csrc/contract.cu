// contract.cu -- aggregation of a level's communities into the next level's
// graph on sm_100a.
//
// Reference semantics (upicine/louvain-community-detection):
//   non-empty flags + renumber by exclusive scan ... aggregation.cu:21-36,
//                                                   389-393
//   vertices grouped by community ................. aggregation.cu:38-45,
//                                                   396-399
//   per-community merge of member edges keyed by
//   neighbour community, weights summed ........... aggregation.cu:57-357
//   new offsets (scan of distinct counts) ......... aggregation.cu:452-456
//   final CSR, neighbour ids renumbered ........... aggregation.cu:359-378
//   louvian.py:163-215 states the same contraction.
//
// Design:
//   * new ids, member offsets and each member's start in the flattened
//     edge space of its community come from scans, so every kernel walks a
//     community's edges as one flat range (load-balanced across members,
//     where the reference walks members one after another).
//   * communities are split by entry count into warp (<= 128 entries,
//     256-slot shared table), block (<= 4096 entries, 8192-slot shared
//     table) and multi-block classes (global table sized from the
//     community's own entry count; the reference sizes every table from the
//     level's vertex count).
//   * neighbour ids are renumbered before hashing (cnew[u]), so rows are
//     emitted in final ids and the last copy is a plain gather.
//   * weights are summed in FP64 and rounded once to FP32.  A row's entries
//     come out in table order; as in the reference (whose order depends on
//     atomicCAS winners) only the set of (neighbour, weight) pairs of a row
//     is defined.
#include <algorithm>
#include <cstring>

#include "lv_internal.h"

namespace lvb {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kWarpSlots = 256;                 // class W table
constexpr int kMidSlots = 2048;                 // class B table
constexpr int kMidSmem = kMidSlots * 12 + kThreads * 16;
constexpr int kBlockSlots = 8192;               // class B2 table
constexpr int kBlockSmem = kBlockSlots * 12 + kThreads * 16;
static_assert(kMergeMidMax * 3 / 2 + 1 <= kMidSlots &&
                  kMergeBlockMax * 3 / 2 + 1 <= kBlockSlots,
              "tables keep load factor <= 2/3");

// Slot from the top bits of a multiplicative (Fibonacci) hash: the low bits
// of key * odd depend only on the key's low bits, and vertex ids such as
// R-MAT's share low-bit patterns, which piled them into a few probe chains.
__device__ __forceinline__ uint32_t hash_slot(uint32_t key, uint32_t mask) {
  return __umulhi(key * 2654435761u, mask + 1u);  // mask + 1: a power of two
}

// Table slots used for a row of d entries: a power of two >= 1.5 d (load
// factor <= 2/3), at most tmax.
__device__ __forceinline__ uint32_t table_size_for(uint32_t d, uint32_t tmax) {
  const uint32_t want = d + (d >> 1) + 1;
  uint32_t t = 32;
  while (t < want) t <<= 1;
  return t < tmax ? t : tmax;
}

__device__ __forceinline__ uint32_t table_insert(uint32_t* keys, uint32_t mask,
                                                 uint32_t key, uint32_t* err) {
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
  atomicExch(err, 1u);
  return 0;
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
  return x;
}

struct Ctx {
  const uint64_t* off;
  const uint32_t* col;
  const float* w;
  const uint32_t* comm_sz;
  const uint32_t* members;
  const uint32_t* mem_off;
  const uint32_t* cnew;
  const uint64_t* mstart;
  const uint32_t* comm_list;
  uint32_t* tcol;
  float* tw;
  uint64_t* new_deg;
  uint32_t* err;
};

// flag_id[c] = comm_sz[c] > 0 ; mem_off[c] = comm_sz[c]  (scanned after)
__global__ void flags_kernel(const uint32_t* comm_sz, uint32_t n,
                             uint32_t* flag_id, uint32_t* mem_off,
                             uint32_t* cursor) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += gridDim.x * blockDim.x) {
    const uint32_t s = comm_sz[c];
    flag_id[c] = s ? 1u : 0u;
    mem_off[c] = s;
    cursor[c] = 0u;
  }
}

// members grouped by community; cnew[v] = new id of comm[v];
// comm_list[new id] = old id.
__global__ void members_kernel(const uint32_t* comm, const uint32_t* comm_sz,
                               uint32_t n, const uint32_t* flag_id,
                               const uint32_t* mem_off, uint32_t* cursor,
                               uint32_t* members, uint32_t* cnew,
                               uint32_t* comm_list) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += gridDim.x * blockDim.x) {
    const uint32_t c = comm[v];
    if (comm_sz[c] == 0u) {  // dropped graph (batched form): no new vertex
      cnew[v] = 0u;
      continue;
    }
    const uint32_t pos = mem_off[c] + atomicAdd(&cursor[c], 1u);
    members[pos] = v;
    cnew[v] = flag_id[c];
    if (comm_sz[v]) comm_list[flag_id[v]] = v;
  }
}

// mstart[i] = degree of members[i] for the *d_members grouped vertices
// (fewer than n when the batched form drops graphs), 0 beyond.
__global__ void member_deg_kernel(const uint64_t* off, const uint32_t* members,
                                  uint32_t n, const uint32_t* d_members,
                                  uint64_t* mstart) {
  const uint32_t nm = *d_members;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= n;
       i += gridDim.x * blockDim.x) {
    uint64_t d = 0;
    if (i < nm) {
      const uint32_t v = members[i];
      d = off[v + 1] - off[v];
    }
    mstart[i] = d;
  }
}

// entries and staging offset of every new community; new_deg zeroed.
// n_upper bounds the new vertex count *d_new_n.
__global__ void comm_deg_kernel(const uint32_t* comm_list, uint32_t n_upper,
                                const uint32_t* d_new_n,
                                const uint32_t* comm_sz, const uint32_t* mem_off,
                                const uint64_t* mstart, uint64_t* comm_deg,
                                uint64_t* seg, uint64_t* new_deg) {
  const uint32_t new_n = *d_new_n;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= n_upper && i <= new_n;
       i += gridDim.x * blockDim.x) {
    new_deg[i] = 0ull;
    if (i < new_n) {
      const uint32_t c = comm_list[i];
      const uint32_t m0 = mem_off[c];
      const uint64_t s = mstart[m0];
      seg[i] = s;
      comm_deg[i] = mstart[m0 + comm_sz[c]] - s;
    }
  }
}

// Class-G plan totals, after the class sizes in counts[0..7] so one copy
// brings both to the host: [10] blocks (kMergeChunk entries each), [12..13]
// table slots (u64).  counts[8..9] hold the new entry count later.
constexpr int kGTotals = 10;

// The class-G plan on the device (one block): every multi-block community
// (counts[7] of them, listed after the warp and block classes in comm_cls)
// gets a global table of a power of two >= 2 min(entries, new n) + 1 slots
// and ceil(entries / kMergeChunk) blocks; table offsets and first blocks
// are exclusive scans.  `cap` is the capacity of the per-community and
// per-block arrays; a level past it writes no plan and leaves the totals
// at ~0 (the host reports it).
__global__ void __launch_bounds__(1024)
    g_plan_kernel(const uint64_t* __restrict__ comm_deg, const uint32_t* __restrict__ comm_cls,
                  uint32_t* counts, uint64_t cap, uint64_t* tab_off, uint32_t* tab_size,
                  uint32_t* blk_first) {
  __shared__ unsigned long long sh[33];
  const uint32_t new_n = counts[0];
  const uint32_t* list = comm_cls + counts[4] + counts[5] + counts[6];
  const uint32_t cnt = counts[7];
  uint64_t* tot64 = reinterpret_cast<uint64_t*>(counts + 12);
  unsigned long long c_slots = 0, c_blk = 0, t;
  bool over = cnt > cap;
  for (uint32_t base = 0; !over && base < cnt; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    unsigned long long T = 0, nch = 0;
    if (i < cnt) {
      const unsigned long long d = comm_deg[list[i]];
      const unsigned long long distinct = d < new_n ? d : new_n;
      T = 1;
      while (T < 2 * distinct + 1) T <<= 1;
      nch = (d + kMergeChunk - 1) / kMergeChunk;
    }
    const unsigned long long x_s = block_exclusive_scan(T, sh, &t);
    const unsigned long long s_s = c_slots;
    c_slots += t;
    const unsigned long long x_b = block_exclusive_scan(nch, sh, &t);
    const unsigned long long s_b = c_blk;
    c_blk += t;
    if (i < cnt) {
      tab_off[i] = s_s + x_s;
      tab_size[i] = (uint32_t)T;
      blk_first[i] = (uint32_t)(s_b + x_b);
    }
    over = c_blk > cap;  // uniform across the block
  }
  if (threadIdx.x == 0) {
    if (over) {
      counts[kGTotals] = ~0u;
      tot64[0] = ~0ull;
    } else {
      blk_first[cnt] = (uint32_t)c_blk;
      counts[kGTotals] = (uint32_t)c_blk;
      tot64[0] = c_slots;
    }
  }
}

// The class-G block map (a warp per community): block -> community index,
// chunk, chunks of the community, packed as blk_comm[b], blk_chunk[b] and
// blk_chunk[nblk + b].
__global__ void g_fill_kernel(const uint32_t* __restrict__ counts,
                              const uint32_t* __restrict__ blk_first, uint32_t* blk_comm,
                              uint32_t* blk_chunk) {
  const uint32_t cnt = counts[7], nblk = counts[kGTotals];
  if (nblk == ~0u) return;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < cnt; i += warps) {
    const uint32_t b0 = blk_first[i], nch = blk_first[i + 1] - b0;
    for (uint32_t ch = lane; ch < nch; ch += 32) {
      blk_comm[b0 + ch] = i;
      blk_chunk[b0 + ch] = ch;
      blk_chunk[nblk + b0 + ch] = nch;
    }
  }
}

// Class W: one warp per community, flattened member edges, 256-slot table.
__global__ void __launch_bounds__(kThreads)
    merge_warp_kernel(Ctx C, const uint32_t* list, uint32_t count) {
  __shared__ double vals_sm[kWarps][kWarpSlots];
  __shared__ uint32_t keys_sm[kWarps][kWarpSlots];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double* vals = vals_sm[wib];
  uint32_t* keys = keys_sm[wib];
  for (uint32_t idx = blockIdx.x * kWarps + wib; idx < count;
       idx += gridDim.x * kWarps) {
    const uint32_t cn = list[idx];
    const uint32_t c = C.comm_list[cn];
    const uint32_t m0 = C.mem_off[c], msz = C.comm_sz[c];
    const uint64_t seg = C.mstart[m0];
    const uint64_t total = C.mstart[m0 + msz] - seg;
    const uint32_t tv = table_size_for((uint32_t)total, kWarpSlots);
    const uint32_t mask = tv - 1;
    for (uint32_t i = lane; i < tv; i += 32) {
      keys[i] = kEmptyKey;
      vals[i] = 0.0;
    }
    __syncwarp();
    // edges into the community itself (most of them, once the moves have
    // converged) are summed in registers instead of one contended slot
    double hot_acc = 0.0;
    bool hot_seen = false;
    for (uint32_t mb = 0; mb < msz; mb += 32) {
      const uint32_t mi = mb + lane;
      const bool mv = mi < msz;
      const uint32_t nvalid = min(32u, msz - mb);
      uint64_t my_start = mv ? C.mstart[m0 + mi] - seg : ~0ull;
      uint64_t my_off = 0;
      if (mv) my_off = C.off[C.members[m0 + mi]];
      const uint64_t lo = __shfl_sync(kFull, my_start, 0);
      const uint64_t hi = (mb + 32 < msz) ? C.mstart[m0 + mb + 32] - seg : total;
      // the batch's entries (at most kMergeWarpMax: a community of this
      // class has no more) in kWaves waves whose loads are all issued
      // before the first insert
      constexpr int kWaves = (int)(kMergeWarpMax / 32);
      uint32_t key[kWaves];
      float wt[kWaves];
#pragma unroll
      for (int k = 0; k < kWaves; k++) {
        key[k] = kEmptyKey;
        wt[k] = 0.0f;
        if (lo + (uint64_t)k * 32 >= hi) continue;  // warp-uniform: most rows are short
        const uint64_t p = lo + (uint64_t)k * 32 + lane;
        // largest member q with start_q <= p
        int klo = 0, khi = (int)nvalid - 1;
#pragma unroll
        for (int it = 0; it < 5; it++) {
          const int mid = (klo + khi + 1) >> 1;
          const uint64_t sm = __shfl_sync(kFull, my_start, mid);
          if (sm <= p) klo = mid; else khi = mid - 1;
          if (khi < klo) khi = klo;
        }
        const uint64_t vo = __shfl_sync(kFull, my_off, klo);
        const uint64_t vs = __shfl_sync(kFull, my_start, klo);
        if (p < hi) {
          const uint64_t j = vo + (p - vs);
          key[k] = C.col[j];
          wt[k] = C.w[j];
        }
      }
#pragma unroll
      for (int k = 0; k < kWaves; k++)
        if (key[k] != kEmptyKey) key[k] = C.cnew[key[k]];
#pragma unroll
      for (int k = 0; k < kWaves; k++) {
        if (key[k] == kEmptyKey) continue;
        if (key[k] == cn) {  // intra-community edge: the new self-loop
          hot_acc += (double)wt[k];
          hot_seen = true;
        } else {  // every lane inserts its own entry: equal keys meet in the CAS
          atomicAdd(&vals[table_insert(keys, mask, key[k], C.err)], (double)wt[k]);
        }
      }
    }
    hot_acc = warp_sum(hot_acc);
    const bool any_hot = __any_sync(kFull, hot_seen);
    __syncwarp();
    if (lane == 0 && any_hot) {
      const uint32_t slot = table_insert(keys, mask, cn, C.err);
      vals[slot] += hot_acc;
    }
    __syncwarp();
    uint32_t cnt = 0;
    for (uint32_t i0 = 0; i0 < tv; i0 += 32) {
      const uint32_t key = keys[i0 + lane];
      const bool occ = key != kEmptyKey;
      const unsigned b = __ballot_sync(kFull, occ);
      if (occ) {
        const uint32_t pos = cnt + __popc(b & ((1u << lane) - 1u));
        C.tcol[seg + pos] = key;
        C.tw[seg + pos] = (float)vals[i0 + lane];
      }
      cnt += __popc(b);
    }
    if (lane == 0) C.new_deg[cn] = cnt;
    __syncwarp();
  }
}

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t x, uint32_t* sm,
                                                    uint32_t* total) {
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  uint32_t incl = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) sm[wib] = incl;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t run = 0;
    for (int i = 0; i < kWarps; i++) {
      uint32_t t = sm[i];
      sm[i] = run;
      run += t;
    }
    sm[kWarps] = run;
  }
  __syncthreads();
  const uint32_t r = sm[wib] + incl - x;
  *total = sm[kWarps];
  __syncthreads();
  return r;
}

// Inserts positions [lo, hi) of a community's flattened edge range into a
// table; members are staged through shared memory 256 at a time.
__device__ __forceinline__ void insert_range(const Ctx& C, uint32_t m0,
                                             uint32_t msz, uint64_t seg,
                                             uint64_t total, uint64_t lo,
                                             uint64_t hi, uint32_t* keys,
                                             double* vals, uint32_t mask,
                                             uint64_t* s_start,
                                             uint64_t* s_off, uint32_t hot,
                                             double& hot_acc, bool& hot_seen) {
  // first member whose range contains lo: largest k with start_k <= lo
  __shared__ uint32_t s_k;
  if (threadIdx.x == 0) {
    uint32_t a = 0, b = msz - 1;
    while (a < b) {
      const uint32_t mid = (a + b + 1) >> 1;
      if (C.mstart[m0 + mid] - seg <= lo) a = mid; else b = mid - 1;
    }
    s_k = a;
  }
  __syncthreads();
  uint32_t k0 = s_k;
  uint64_t pos = lo;
  while (pos < hi) {
    const uint32_t kk = k0 + threadIdx.x;
    if (kk < msz) {
      s_start[threadIdx.x] = C.mstart[m0 + kk] - seg;
      s_off[threadIdx.x] = C.off[C.members[m0 + kk]];
    } else {
      s_start[threadIdx.x] = ~0ull;
      s_off[threadIdx.x] = 0;
    }
    __syncthreads();
    const uint32_t nvalid = min((uint32_t)kThreads, msz - k0);
    const uint64_t chunk_end =
        (k0 + kThreads < msz) ? min(hi, C.mstart[m0 + k0 + kThreads] - seg) : hi;
    // kWaves waves of the block at a time, every load of a batch issued
    // before its first insert
    constexpr int kWaves = 4;
    for (uint64_t p0 = pos; p0 < chunk_end; p0 += (uint64_t)kWaves * kThreads) {
      uint32_t key[kWaves];
      float wt[kWaves];
#pragma unroll
      for (int k = 0; k < kWaves; k++) {
        const uint64_t p = p0 + (uint64_t)k * kThreads + threadIdx.x;
        key[k] = kEmptyKey;
        wt[k] = 0.0f;
        if (p0 + (uint64_t)k * kThreads >= chunk_end) continue;  // block-uniform
        if (p < chunk_end) {
          int a = 0, b = (int)nvalid - 1;
          while (a < b) {
            const int mid = (a + b + 1) >> 1;
            if (s_start[mid] <= p) a = mid; else b = mid - 1;
          }
          const uint64_t j = s_off[a] + (p - s_start[a]);
          key[k] = C.col[j];
          wt[k] = C.w[j];
        }
      }
#pragma unroll
      for (int k = 0; k < kWaves; k++)
        if (key[k] != kEmptyKey) key[k] = C.cnew[key[k]];
#pragma unroll
      for (int k = 0; k < kWaves; k++) {
        if (key[k] == kEmptyKey) continue;
        if (key[k] == hot) {
          hot_acc += (double)wt[k];
          hot_seen = true;
        } else {
          atomicAdd(&vals[table_insert(keys, mask, key[k], C.err)], (double)wt[k]);
        }
      }
    }
    pos = chunk_end;
    k0 += kThreads;
    __syncthreads();
  }
  (void)total;
}

// Classes B (SLOTS = 2048: <= 1024 entries) and B2 (8192: <= 4096): one
// block per community, shared table of up to SLOTS slots.
template <int SLOTS>
__global__ void __launch_bounds__(kThreads)
    merge_block_kernel(Ctx C, const uint32_t* list, uint32_t count) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* vals = reinterpret_cast<double*>(smem_raw);
  uint64_t* s_start = reinterpret_cast<uint64_t*>(smem_raw + SLOTS * 8);
  uint64_t* s_off = s_start + kThreads;
  uint32_t* keys = reinterpret_cast<uint32_t*>(smem_raw + SLOTS * 8 + kThreads * 16);
  __shared__ uint32_t scan_sm[kWarps + 1];
  for (uint32_t idx = blockIdx.x; idx < count; idx += gridDim.x) {
    const uint32_t cn = list[idx];
    const uint32_t c = C.comm_list[cn];
    const uint32_t m0 = C.mem_off[c], msz = C.comm_sz[c];
    const uint64_t seg = C.mstart[m0];
    const uint64_t total = C.mstart[m0 + msz] - seg;
    // class B rows hold > 128 entries, so tv >= 256 = kThreads
    const uint32_t tv = table_size_for((uint32_t)total, SLOTS);
    for (uint32_t i = threadIdx.x; i < tv; i += kThreads) {
      keys[i] = kEmptyKey;
      vals[i] = 0.0;
    }
    __syncthreads();
    double hot_acc = 0.0;
    bool hot_seen = false;
    insert_range(C, m0, msz, seg, total, 0, total, keys, vals, tv - 1, s_start, s_off, cn,
                 hot_acc, hot_seen);
    // every warp adds its share of the new self-loop (FP64 sums of FP32
    // weights are exact in any order): no block-wide sum first
    hot_acc = warp_sum(hot_acc);
    if (__any_sync(kFull, hot_seen) && (threadIdx.x & 31) == 0)
      atomicAdd(&vals[table_insert(keys, tv - 1, cn, C.err)], hot_acc);
    __syncthreads();
    // emit: thread t owns slots [t*per, t*per + per)
    const uint32_t per = tv / kThreads;
    uint32_t local = 0;
    for (uint32_t i = 0; i < per; i++) local += keys[threadIdx.x * per + i] != kEmptyKey;
    uint32_t tot;
    uint32_t pos = block_excl_scan(local, scan_sm, &tot);
    for (uint32_t i = 0; i < per; i++) {
      const uint32_t sl = threadIdx.x * per + i;
      const uint32_t key = keys[sl];
      if (key != kEmptyKey) {
        C.tcol[seg + pos] = key;
        C.tw[seg + pos] = (float)vals[sl];
        pos++;
      }
    }
    if (threadIdx.x == 0) C.new_deg[cn] = tot;
    __syncthreads();
  }
}

struct GArgs {
  const uint32_t* list;      // class G new ids
  const uint64_t* tab_off;   // per class-G index
  const uint32_t* tab_size;  // per class-G index (power of two)
  const uint32_t* blk_comm;  // per block: class-G index
  const uint32_t* blk_chunk; // per block: chunk index
  const uint32_t* blk_nchunks;
  uint32_t* keys;
  double* vals;
  uint32_t nblocks;
};

// Class G: blocks insert chunks of a community's flattened range into its
// global table.
__global__ void __launch_bounds__(kThreads)
    merge_global_insert_kernel(Ctx C, GArgs G) {
  __shared__ uint64_t s_start[kThreads];
  __shared__ uint64_t s_off[kThreads];
  for (uint32_t b = blockIdx.x; b < G.nblocks; b += gridDim.x) {
    const uint32_t gi = G.blk_comm[b], ch = G.blk_chunk[b];
    const uint32_t cn = G.list[gi];
    const uint32_t c = C.comm_list[cn];
    const uint32_t m0 = C.mem_off[c], msz = C.comm_sz[c];
    const uint64_t seg = C.mstart[m0];
    const uint64_t total = C.mstart[m0 + msz] - seg;
    const uint64_t lo = (uint64_t)ch * kMergeChunk;
    const uint64_t hi = min(total, lo + kMergeChunk);
    uint32_t* keys = G.keys + G.tab_off[gi];
    double* vals = G.vals + G.tab_off[gi];
    const uint32_t mask = G.tab_size[gi] - 1;
    double hot_acc = 0.0;
    bool hot_seen = false;
    insert_range(C, m0, msz, seg, total, lo, hi, keys, vals, mask, s_start, s_off, cn,
                 hot_acc, hot_seen);
    hot_acc = warp_sum(hot_acc);  // per warp, as in merge_block_kernel
    if (__any_sync(kFull, hot_seen) && (threadIdx.x & 31) == 0)
      atomicAdd(&vals[table_insert(keys, mask, cn, C.err)], hot_acc);
    __syncthreads();
  }
}

// Class G: blocks compact slices of the tables into the staging rows.
__global__ void __launch_bounds__(kThreads)
    merge_global_emit_kernel(Ctx C, GArgs G) {
  __shared__ uint32_t scan_sm[kWarps + 1];
  __shared__ uint32_t base_sm;
  for (uint32_t b = blockIdx.x; b < G.nblocks; b += gridDim.x) {
    const uint32_t gi = G.blk_comm[b], ch = G.blk_chunk[b];
    const uint32_t nch = G.blk_nchunks[b];
    const uint32_t cn = G.list[gi];
    const uint32_t c = C.comm_list[cn];
    const uint64_t seg = C.mstart[C.mem_off[c]];
    const uint64_t T = G.tab_size[gi];
    const uint64_t s0 = T * ch / nch, s1 = T * (ch + 1) / nch;
    const uint32_t* keys = G.keys + G.tab_off[gi];
    const double* vals = G.vals + G.tab_off[gi];
    for (uint64_t i0 = s0; i0 < s1; i0 += kThreads) {
      const uint64_t i = i0 + threadIdx.x;
      const bool occ = i < s1 && keys[i] != kEmptyKey;
      uint32_t tot;
      const uint32_t r = block_excl_scan(occ ? 1u : 0u, scan_sm, &tot);
      if (threadIdx.x == 0 && tot)
        base_sm = (uint32_t)atomicAdd((unsigned long long*)&C.new_deg[cn],
                                      (unsigned long long)tot);
      __syncthreads();
      if (occ) {
        const uint64_t pos = seg + base_sm + r;
        C.tcol[pos] = keys[i];
        C.tw[pos] = (float)vals[i];
      }
      __syncthreads();
    }
  }
}

// Final CSR: row cn copied from its staging range to new offsets.  Rows are
// dealt round robin to the warps (consecutive new ids -- often the large
// communities formed around hubs -- land on different warps); a warp takes
// 32 of its rows at a time, every lane loading one row's bounds, then
// copies them one after another, 32 entries per store.  Rows longer than
// kLongRow entries (only communities of the largest class have them) are
// left to compress_long_kernel, where the whole grid copies each.
constexpr uint64_t kLongRow = kMergeBlockMax;
__global__ void __launch_bounds__(kThreads)
    compress_kernel(const uint64_t* __restrict__ seg, const uint64_t* __restrict__ new_off,
                    uint32_t new_n, const uint32_t* __restrict__ tcol,
                    const float* __restrict__ tw, uint32_t* __restrict__ out_col,
                    float* __restrict__ out_w) {
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint64_t nwarps = (uint64_t)gridDim.x * kWarps;
  const uint64_t w = (uint64_t)blockIdx.x * kWarps + wib;
  for (uint64_t k0 = 0; w + k0 * nwarps < new_n; k0 += 32) {
    const uint64_t cn = w + (k0 + lane) * nwarps;
    uint64_t dst = 0, cnt = 0, src = 0;
    if (cn < new_n) {
      dst = new_off[cn];
      cnt = new_off[cn + 1] - dst;
      src = seg[cn];
      if (cnt > kLongRow) cnt = 0;
    }
    for (int i = 0; i < 32; i++) {
      const uint64_t di = __shfl_sync(kFull, dst, i), ci = __shfl_sync(kFull, cnt, i);
      const uint64_t si = __shfl_sync(kFull, src, i);
      // four loads in flight per lane (the staging and the output do not
      // overlap), so a long row is not one round trip per 32 entries
      for (uint64_t j0 = 0; j0 < ci; j0 += 128) {
        uint32_t c[4];
        float w[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const uint64_t j = j0 + (uint64_t)k * 32 + lane;
          if (j < ci) {
            c[k] = tcol[si + j];
            w[k] = tw[si + j];
          }
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const uint64_t j = j0 + (uint64_t)k * 32 + lane;
          if (j < ci) {
            out_col[di + j] = c[k];
            out_w[di + j] = w[k];
          }
        }
      }
    }
  }
}

// The long rows: every class-G community's row of more than kLongRow
// entries, a block per row (rows dealt round robin to the blocks), four
// loads in flight per thread.  (The whole grid copying one row after
// another left most threads idle on R-MAT's thousands of long rows: 15.6
// of R-MAT 24's 51 ms level-0 contraction.)
__global__ void __launch_bounds__(kThreads)
    compress_long_kernel(const uint32_t* __restrict__ glist, uint32_t count,
                         const uint64_t* __restrict__ seg, const uint64_t* __restrict__ new_off,
                         const uint32_t* __restrict__ tcol, const float* __restrict__ tw,
                         uint32_t* __restrict__ out_col, float* __restrict__ out_w) {
  for (uint32_t i = blockIdx.x; i < count; i += gridDim.x) {
    const uint32_t cn = glist[i];
    const uint64_t dst = new_off[cn];
    const uint64_t cnt = new_off[cn + 1] - dst;
    if (cnt <= kLongRow) continue;  // block-uniform: compress_kernel's
    const uint64_t src = seg[cn];
    for (uint64_t j0 = 0; j0 < cnt; j0 += 4 * kThreads) {
      uint32_t c[4];
      float w[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const uint64_t j = j0 + (uint64_t)k * kThreads + threadIdx.x;
        if (j < cnt) {
          c[k] = tcol[src + j];
          w[k] = tw[src + j];
        }
      }
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const uint64_t j = j0 + (uint64_t)k * kThreads + threadIdx.x;
        if (j < cnt) {
          out_col[dst + j] = c[k];
          out_w[dst + j] = w[k];
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Contraction by sorting: every entry (u, v) gets the key
// (new id of comm(u), new id of comm(v)); a stable radix sort brings equal
// keys together, a segmented reduction sums their weights (FP64, rounded
// once) and the sorted row ids give the new offsets.  Rows come out sorted
// by column.
// ---------------------------------------------------------------------------
__global__ void cnew_kernel(const uint32_t* __restrict__ comm, const uint32_t* __restrict__ new_id,
                            uint32_t n, uint32_t* __restrict__ cnew) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    cnew[v] = new_id[comm[v]];
}

__global__ void sort_keys_kernel(const uint32_t* __restrict__ rowid,
                                 const uint32_t* __restrict__ col,
                                 const uint32_t* __restrict__ cnew, uint64_t nnz, int bits,
                                 uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < nnz;
       j += (uint64_t)gridDim.x * blockDim.x) {
    keys[j] = ((uint64_t)cnew[rowid[j]] << bits) | cnew[col[j]];
    vals[j] = (uint32_t)j;
  }
}

__global__ void heads_kernel(const uint64_t* __restrict__ keys, uint64_t nnz,
                             uint32_t* __restrict__ heads) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < nnz;
       j += (uint64_t)gridDim.x * blockDim.x)
    heads[j] = (j == 0 || keys[j] != keys[j - 1]) ? 1u : 0u;
}

__global__ void zero_f64_kernel(double* a, const uint32_t* d_count, uint64_t cap) {
  const uint64_t n = min((uint64_t)*d_count, cap);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    a[i] = 0.0;
}

// Run r(j) = heads up to j - 1.  Weights of a run are summed in the warp
// (runs are contiguous) and once per warp segment into acc[r]; FP64 sums of
// FP32 weights are exact whatever the order.  Heads write the new entry's
// column and row.
__global__ void __launch_bounds__(256)
    run_reduce_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                      const uint32_t* __restrict__ heads, const uint32_t* __restrict__ pos,
                      uint64_t nnz, const float* __restrict__ w, int bits,
                      double* __restrict__ acc, uint32_t* __restrict__ out_col,
                      uint32_t* __restrict__ row_of) {
  const int lane = threadIdx.x & 31;
  const uint64_t mask = (1ull << bits) - 1ull;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t j0 = blockIdx.x * (uint64_t)blockDim.x; j0 < nnz; j0 += stride) {
    const uint64_t j = j0 + threadIdx.x;  // whole warps iterate together
    const bool valid = j < nnz;
    uint32_t r = 0xFFFFFFFFu;
    double x = 0.0;
    if (valid) {
      const uint32_t h = heads[j];
      r = pos[j] + h - 1u;
      x = (double)w[vals[j]];
      if (h) {
        const uint64_t k = keys[j];
        out_col[r] = (uint32_t)(k & mask);
        row_of[r] = (uint32_t)(k >> bits);
      }
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const double y = __shfl_down_sync(kFull, x, o);
      const uint32_t ry = __shfl_down_sync(kFull, r, o);
      if (lane + o < 32 && ry == r) x += y;
    }
    const uint32_t rp = __shfl_up_sync(kFull, r, 1);
    if (valid && (lane == 0 || rp != r)) atomicAdd(&acc[r], x);
  }
}

// off[v] = first new entry of row >= v for v in [0, n_rows]; the entry count
// is read on the device.
__global__ void bounds_dev_kernel(const uint32_t* __restrict__ row_of, const uint32_t* d_total,
                                  uint64_t cap, uint32_t n_rows, uint64_t* __restrict__ off) {
  const uint64_t total = min((uint64_t)*d_total, cap);
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j <= total;
       j += (uint64_t)gridDim.x * blockDim.x) {
    const int64_t prev = j ? (int64_t)row_of[j - 1] : -1;
    const uint32_t cur = j < total ? row_of[j] : n_rows;
    for (int64_t v = prev + 1; v <= (int64_t)cur && v <= (int64_t)n_rows; v++) off[v] = j;
  }
}

__global__ void round_f64_kernel(const double* __restrict__ acc, const uint32_t* d_count,
                                 uint64_t cap, float* __restrict__ out) {
  const uint64_t n = min((uint64_t)*d_count, cap);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = (float)acc[i];
}

int bits_of(uint64_t max_value) {
  int b = 0;
  while (b < 64 && (max_value >> b)) b++;
  return b;
}

unsigned gridcap(uint64_t work, unsigned per_sm) {
  const uint64_t cap = (uint64_t)sm_count_cached() * per_sm;
  if (work == 0) return 1;
  return (unsigned)(work < cap ? work : cap);
}

}  // namespace

cudaError_t configure_contract_kernels() {
  cudaError_t e = cudaFuncSetAttribute(merge_block_kernel<kMidSlots>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kMidSmem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(merge_block_kernel<kBlockSlots>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, kBlockSmem);
}

#define LV_TRY(x)                              \
  do {                                         \
    cudaError_t e_ = (x);                      \
    if (e_ != cudaSuccess) return e_;          \
  } while (0)

namespace {

// The class-G plan on the device with arrays of capacity >= cap: table
// offsets and sizes, first block of every community, the block map.
cudaError_t plan_g(ContractBuffers& B, uint64_t nnz, uint64_t cap, cudaStream_t st,
                   cudaError_t (*grow)(void*, size_t, size_t), void* grow_ctx) {
  if (cap > B.g_cap) LV_TRY(grow(grow_ctx, 0, cap));
  (count_launches(1), g_plan_kernel<<<1, 1024, 0, st>>>(B.comm_deg, B.comm_cls, B.counts,
                                                        B.g_cap, B.g_tab_off, B.g_tab_size,
                                                        B.g_blk_first));
  LV_TRY(cudaGetLastError());
  (count_launches(1), g_fill_kernel<<<gridcap((nnz / (kMergeBlockMax + 1) + 8) / 8, 8),
                                      kThreads, 0, st>>>(B.counts, B.g_blk_first, B.g_blk_comm,
                                                         B.g_blk_chunk));
  return cudaGetLastError();
}

// The class-G arrays hold the plan when they have room for the most a
// level of nnz entries can need: a class-G community has more than
// kMergeBlockMax entries and its blocks cover its entries in kMergeChunk
// pieces, of the level's nnz in all.
uint64_t g_bound_of(uint64_t nnz) { return nnz / (kMergeBlockMax + 1) + nnz / kMergeChunk + 1; }

}  // namespace

cudaError_t contract_front(const LevelView& L, uint64_t nnz, ContractBuffers& B,
                           ScanScratch& S, cudaStream_t st,
                           cudaError_t (*grow)(void*, size_t, size_t), void* grow_ctx) {
  const uint32_t n = L.n;
  const unsigned g1 = gridcap((n + 255) / 256, 8);
  (count_launches(1), flags_kernel<<<g1, 256, 0, st>>>(L.comm_sz, n, B.flag_id, B.mem_off, B.cursor));
  LV_TRY(cudaGetLastError());
  LV_TRY(exclusive_scan_u32(B.flag_id, B.flag_id, n, B.counts + 0, S, st));
  LV_TRY(exclusive_scan_u32(B.mem_off, B.mem_off, n, B.counts + 1, S, st));
  (count_launches(1), members_kernel<<<g1, 256, 0, st>>>(L.comm, L.comm_sz, n, B.flag_id, B.mem_off,
                                     B.cursor, B.members, B.cnew, B.comm_list));
  LV_TRY(cudaGetLastError());
  (count_launches(1), member_deg_kernel<<<gridcap((n + 256) / 256, 8), 256, 0, st>>>(
      L.off, B.members, n, B.counts + 1, B.mstart));
  LV_TRY(cudaGetLastError());
  LV_TRY(exclusive_scan_u64(B.mstart, B.mstart, (size_t)n + 1, nullptr, S, st));
  // sizes of the new communities and their classes, with the new vertex
  // count read on the device (no host round trip before the merges)
  (count_launches(1), comm_deg_kernel<<<gridcap((n + 256) / 256, 8), 256, 0, st>>>(
      B.comm_list, n, B.counts + 0, L.comm_sz, B.mem_off, B.mstart, B.comm_deg,
      B.seg, B.new_deg));
  LV_TRY(cudaGetLastError());
  LV_TRY(partition_by_size4(B.comm_deg, n, B.counts + 0, kMergeWarpMax, kMergeMidMax,
                            kMergeBlockMax, B.comm_cls, B.counts + 4, B.tmp, S, st));
  // class-G plan on the device, its totals copied with the class sizes
  if (nnz > kMergeBlockMax) LV_TRY(plan_g(B, nnz, g_bound_of(nnz), st, grow, grow_ctx));
  return cudaMemcpyAsync(B.host_counts, B.counts, 16 * sizeof(uint32_t),
                         cudaMemcpyDeviceToHost, st);
}

cudaError_t contract_back(const LevelView& L, uint64_t nnz, ContractBuffers& B,
                          ScanScratch& S, uint64_t* out_off, uint32_t* out_col,
                          float* out_w, ContractResult* res, cudaStream_t st,
                          cudaError_t (*grow)(void*, size_t, size_t), void* grow_ctx,
                          bool defer_total) {
  uint32_t* h_counts = B.host_counts;
  const bool g_planned = nnz > kMergeBlockMax;
  const uint32_t new_n = h_counts[0];
  const uint32_t cntW = h_counts[4], cntM = h_counts[5], cntB2 = h_counts[6];
  const uint32_t cntB = cntM + cntB2;  // both block classes
  const uint32_t cntG = h_counts[7];
  // the bound holds when nnz is the level's entry count; otherwise plan
  // again with twice the room until the plan fits
  for (int tries = 0; cntG && (!g_planned || h_counts[kGTotals] == ~0u); tries++) {
    if (tries == 40) return cudaErrorInvalidValue;
    LV_TRY(plan_g(B, nnz, std::max<uint64_t>(2 * (uint64_t)B.g_cap, (uint64_t)cntG + 1), st,
                  grow, grow_ctx));
    LV_TRY(cudaMemcpyAsync(h_counts, B.counts, 16 * sizeof(uint32_t),
                           cudaMemcpyDeviceToHost, st));
    LV_TRY(counted_sync(st));
    if (h_counts[kGTotals] != ~0u) break;
  }

  Ctx C;
  C.off = L.off;
  C.col = L.col;
  C.w = L.w;
  C.comm_sz = L.comm_sz;
  C.members = B.members;
  C.mem_off = B.mem_off;
  C.cnew = B.cnew;
  C.mstart = B.mstart;
  C.comm_list = B.comm_list;
  C.tcol = B.tcol;
  C.tw = B.tw;
  C.new_deg = B.new_deg;
  C.err = &L.sc->error;

  if (cntW) {
    (count_launches(1), merge_warp_kernel<<<gridcap((cntW + kWarps - 1) / kWarps, 4), kThreads, 0, st>>>(
        C, B.comm_cls, cntW));
    LV_TRY(cudaGetLastError());
  }
  if (cntM) {
    (count_launches(1), merge_block_kernel<kMidSlots><<<gridcap(cntM, 7), kThreads, kMidSmem, st>>>(
        C, B.comm_cls + cntW, cntM));
    LV_TRY(cudaGetLastError());
  }
  if (cntB2) {
    (count_launches(1), merge_block_kernel<kBlockSlots><<<gridcap(cntB2, 2), kThreads, kBlockSmem, st>>>(
        C, B.comm_cls + cntW + cntM, cntB2));
    LV_TRY(cudaGetLastError());
  }
  if (cntG) {
    // class-G tables and blocks as planned on the device (few, very large
    // rows); only the table's size is needed here
    const size_t nblk = h_counts[kGTotals];
    uint64_t slots = 0;
    memcpy(&slots, h_counts + kGTotals + 2, sizeof(uint64_t));
    if (slots > B.table_cap) LV_TRY(grow(grow_ctx, slots, 0));
    LV_TRY(cudaMemsetAsync(B.keys, 0xFF, slots * sizeof(uint32_t), st));
    LV_TRY(cudaMemsetAsync(B.vals, 0, slots * sizeof(double), st));
    GArgs G;
    G.list = B.comm_cls + cntW + cntB;
    G.tab_off = B.g_tab_off;
    G.tab_size = B.g_tab_size;
    G.blk_comm = B.g_blk_comm;
    G.blk_chunk = B.g_blk_chunk;
    G.blk_nchunks = B.g_blk_chunk + nblk;
    G.keys = B.keys;
    G.vals = B.vals;
    G.nblocks = (uint32_t)nblk;
    (count_launches(1), merge_global_insert_kernel<<<gridcap(nblk, 8), kThreads, 0, st>>>(C, G));
    LV_TRY(cudaGetLastError());
    (count_launches(1), merge_global_emit_kernel<<<gridcap(nblk, 8), kThreads, 0, st>>>(C, G));
    LV_TRY(cudaGetLastError());
  }
  // new offsets: exclusive scan of the n'+1 counts (last one is 0)
  uint64_t* d_total = reinterpret_cast<uint64_t*>(B.counts + 8);
  LV_TRY(exclusive_scan_u64(B.new_deg, out_off, (size_t)new_n + 1, d_total, S, st));
  (count_launches(1), compress_kernel<<<gridcap(((uint64_t)new_n + kWarps - 1) / kWarps, 8), kThreads, 0, st>>>(
      B.seg, out_off, new_n, B.tcol, B.tw, out_col, out_w));
  LV_TRY(cudaGetLastError());
  if (cntG) {
    (count_launches(1), compress_long_kernel<<<gridcap(1u << 20, 8), kThreads, 0, st>>>(
        B.comm_cls + cntW + cntB, cntG, B.seg, out_off, B.tcol, B.tw, out_col, out_w));
    LV_TRY(cudaGetLastError());
  }
  res->new_n = new_n;
  if (defer_total) {  // the caller reads B.counts + 8 at its next sync
    res->new_nnz = ~0ull;
    return cudaSuccess;
  }
  uint64_t* h_total = reinterpret_cast<uint64_t*>(h_counts + 8);  // pinned
  LV_TRY(cudaMemcpyAsync(h_total, d_total, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  LV_TRY(counted_sync(st));
  res->new_nnz = *h_total;
  return cudaSuccess;
}

cudaError_t contract_level(const LevelView& L, uint64_t nnz,
                           ContractBuffers& B, ScanScratch& S,
                           uint64_t* out_off, uint32_t* out_col, float* out_w,
                           ContractResult* res, cudaStream_t st,
                           cudaError_t (*grow)(void*, size_t, size_t),
                           void* grow_ctx, bool defer_total) {
  LV_TRY(contract_front(L, nnz, B, S, st, grow, grow_ctx));
  LV_TRY(counted_sync(st));
  return contract_back(L, nnz, B, S, out_off, out_col, out_w, res, st, grow, grow_ctx,
                       defer_total);
}

cudaError_t contract_level_sort(const LevelView& L, uint64_t nnz, ContractBuffers& B,
                                SortBuffers& SB, ScanScratch& S, uint64_t* out_off,
                                uint32_t* out_col, float* out_w, ContractResult* res,
                                cudaStream_t st) {
  const uint32_t n = L.n;
  uint32_t* h_counts = B.host_counts;
  const unsigned gv = gridcap((n + 255) / 256, 8);
  const unsigned ge = gridcap((nnz + 255) / 256, 8);
  // renumbering as the hash path (aggregation.cu:389-393)
  (count_launches(1), flags_kernel<<<gv, 256, 0, st>>>(L.comm_sz, n, B.flag_id, B.mem_off, B.cursor));
  LV_TRY(cudaGetLastError());
  LV_TRY(exclusive_scan_u32(B.flag_id, B.flag_id, n, B.counts + 0, S, st));
  (count_launches(1), cnew_kernel<<<gv, 256, 0, st>>>(L.comm, B.flag_id, n, B.cnew));
  LV_TRY(cudaGetLastError());
  // keys of every entry; the level's row ids first (the contraction's
  // column scratch holds no other data at this point)
  uint32_t* rowid = B.tcol;
  LV_TRY(launch_row_ids(L.off, n, nnz, rowid, st));
  const int bits = std::max(1, bits_of(n ? n - 1 : 0));
  if (nnz) {
    (count_launches(1), sort_keys_kernel<<<ge, 256, 0, st>>>(rowid, L.col, B.cnew, nnz, bits,
                                                             SB.keys[0], SB.vals[0]));
    LV_TRY(cudaGetLastError());
  }
  bool alt = false;
  LV_TRY(radix_sort_pairs<uint64_t>(SB.keys[0], SB.vals[0], SB.keys[1], SB.vals[1], nnz, 2 * bits,
                                    SB.counts, SB.scan, st, &alt));
  const uint64_t* keys = SB.keys[alt ? 1 : 0];
  const uint32_t* vals = SB.vals[alt ? 1 : 0];
  double* acc = reinterpret_cast<double*>(SB.keys[alt ? 0 : 1]);  // the idle key buffer
  uint32_t* heads = SB.vals[alt ? 0 : 1];                         // the idle value buffer
  uint32_t* row_of = reinterpret_cast<uint32_t*>(B.tw);
  uint32_t* d_new_nnz = B.counts + 2;
  if (nnz) {
    (count_launches(1), heads_kernel<<<ge, 256, 0, st>>>(keys, nnz, heads));
    LV_TRY(cudaGetLastError());
    LV_TRY(exclusive_scan_u32(heads, SB.pos, nnz, d_new_nnz, SB.scan, st));
    (count_launches(1), zero_f64_kernel<<<ge, 256, 0, st>>>(acc, d_new_nnz, nnz));
    LV_TRY(cudaGetLastError());
    (count_launches(1), run_reduce_kernel<<<ge, 256, 0, st>>>(keys, vals, heads, SB.pos, nnz, L.w,
                                                              bits, acc, out_col, row_of));
    LV_TRY(cudaGetLastError());
  } else {
    LV_TRY(cudaMemsetAsync(d_new_nnz, 0, sizeof(uint32_t), st));
  }
  // new offsets over the old vertex count: rows past the new count are
  // empty and sit beyond the new CSR's n'+1 offsets
  (count_launches(1), bounds_dev_kernel<<<gridcap((nnz + 256) / 256, 8), 256, 0, st>>>(
                          row_of, d_new_nnz, nnz, n, out_off));
  LV_TRY(cudaGetLastError());
  (count_launches(1), round_f64_kernel<<<ge, 256, 0, st>>>(acc, d_new_nnz, nnz, out_w));
  LV_TRY(cudaGetLastError());
  LV_TRY(cudaMemcpyAsync(h_counts, B.counts, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  LV_TRY(counted_sync(st));
  res->new_n = h_counts[0];
  res->new_nnz = h_counts[2];
  return cudaSuccess;
}

}  // namespace lvb
