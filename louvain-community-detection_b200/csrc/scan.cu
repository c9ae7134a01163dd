// scan.cu -- exclusive scans and stable small-key partitions (sm_100a).
//
// These replace the reference's Thrust calls on the level set-up path:
// thrust::partition (modularity.cu:468, aggregation.cu:410; unstable, one
// partition per bucket per pass, each with a host read-back) becomes one
// stable multi-way partition per level; thrust::exclusive_scan /
// inclusive_scan / reduce (aggregation.cu:390-397,452-456) become the
// tile scans below.
#include "lv_internal.h"

namespace lvb {
namespace {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kTile = kScanThreads * kScanItems;  // 4096 elements per block

template <typename T>
__device__ __forceinline__ T warp_inclusive(T x, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

// Exclusive scan of a thread's ITEMS values across the block; returns the
// block total.  Requires blockDim.x == THREADS (<= 1024).
template <typename T, int THREADS, int ITEMS>
__device__ __forceinline__ T block_exclusive(T (&v)[ITEMS], T* warp_sums) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  T local = 0;
#pragma unroll
  for (int i = 0; i < ITEMS; i++) {
    T x = v[i];
    v[i] = local;
    local += x;
  }
  T incl = warp_inclusive(local, lane);
  if (lane == 31) warp_sums[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    T t = (lane < THREADS / 32) ? warp_sums[lane] : T(0);
    t = warp_inclusive(t, lane);
    if (lane < THREADS / 32) warp_sums[lane] = t;
  }
  __syncthreads();
  T prefix = (wid > 0 ? warp_sums[wid - 1] : T(0)) + incl - local;
  T total = warp_sums[THREADS / 32 - 1];
#pragma unroll
  for (int i = 0; i < ITEMS; i++) v[i] += prefix;
  __syncthreads();
  return total;
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads)
    scan_tiles_kernel(const T* in, T* out, size_t n, T* tile_sums, T* single_total) {
  __shared__ T warp_sums[kScanThreads / 32];
  const size_t base = (size_t)blockIdx.x * kTile + (size_t)threadIdx.x * kScanItems;
  T v[kScanItems];
#pragma unroll
  for (int i = 0; i < kScanItems; i++) v[i] = (base + i < n) ? in[base + i] : T(0);
  T total = block_exclusive<T, kScanThreads, kScanItems>(v, warp_sums);
#pragma unroll
  for (int i = 0; i < kScanItems; i++)
    if (base + i < n) out[base + i] = v[i];
  if (threadIdx.x == 0) {
    tile_sums[blockIdx.x] = total;
    if (single_total) *single_total = total;  // a one-tile scan's total
  }
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads)
    scan_add_kernel(T* out, size_t n, const T* tile_prefix) {
  const T add = tile_prefix[blockIdx.x];
  const size_t base = (size_t)blockIdx.x * kTile + (size_t)threadIdx.x * kScanItems;
#pragma unroll
  for (int i = 0; i < kScanItems; i++)
    if (base + i < n) out[base + i] += add;
}

template <typename T>
__global__ void zero_scalar_kernel(T* dst) {
  *dst = T(0);
}

size_t tiles_of(size_t n) { return (n + kTile - 1) / kTile; }

template <typename T>
cudaError_t scan_rec(const T* in, T* out, size_t n, T* total, T* scratch,
                     size_t scratch_elems, cudaStream_t st) {
  if (n == 0) {
    if (total) (count_launches(1), zero_scalar_kernel<T><<<1, 1, 0, st>>>(total));
    return cudaGetLastError();
  }
  const size_t nt = tiles_of(n);
  if (nt > scratch_elems) return cudaErrorInvalidValue;
  T* sums = scratch;
  (count_launches(1), scan_tiles_kernel<T><<<(unsigned)nt, kScanThreads, 0, st>>>(
                          in, out, n, sums, nt == 1 ? total : nullptr));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (nt == 1) return cudaSuccess;
  e = scan_rec<T>(sums, sums, nt, total, scratch + nt, scratch_elems - nt, st);
  if (e != cudaSuccess) return e;
  (count_launches(1), scan_add_kernel<T><<<(unsigned)nt, kScanThreads, 0, st>>>(out, n, sums));
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Stable partition by a small class id (NC <= 9 classes).
// One item per thread, 1024 threads per block.  counts is class-major:
// counts[c * nblocks + b].
// ---------------------------------------------------------------------------
constexpr int kPartThreads = 1024;

template <int NC, class ClassFn>
__global__ void __launch_bounds__(kPartThreads)
    part_count_kernel(uint32_t n, ClassFn fn, uint32_t* counts,
                      uint32_t nblocks) {
  __shared__ uint32_t c_sm[NC];
  if (threadIdx.x < NC) c_sm[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t i = blockIdx.x * kPartThreads + threadIdx.x;
  const int lane = threadIdx.x & 31;
  int c = (i < n) ? fn(i) : -1;
#pragma unroll
  for (int cc = 0; cc < NC; cc++) {
    unsigned b = __ballot_sync(0xffffffffu, c == cc);
    if (lane == 0 && b) atomicAdd(&c_sm[cc], (uint32_t)__popc(b));
  }
  __syncthreads();
  if (threadIdx.x < NC) counts[threadIdx.x * nblocks + blockIdx.x] = c_sm[threadIdx.x];
}

template <int NC, class ClassFn, class ValueFn>
__global__ void __launch_bounds__(kPartThreads)
    part_scatter_kernel(uint32_t n, ClassFn fn, ValueFn val,
                        const uint32_t* offsets, uint32_t nblocks,
                        uint32_t* out, const uint32_t* grand_total,
                        uint32_t* cls_count) {
  constexpr int W = kPartThreads / 32;
  __shared__ uint32_t wc[NC][W];
  if (blockIdx.x == 0 && threadIdx.x < NC) {  // the class sizes
    const int c = threadIdx.x;
    const uint32_t start = offsets[c * nblocks];
    const uint32_t end = (c + 1 < NC) ? offsets[(c + 1) * nblocks] : *grand_total;
    cls_count[c] = end - start;
  }
  const uint32_t i = blockIdx.x * kPartThreads + threadIdx.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int c = (i < n) ? fn(i) : -1;
  unsigned mine = 0;
#pragma unroll
  for (int cc = 0; cc < NC; cc++) {
    unsigned b = __ballot_sync(0xffffffffu, c == cc);
    if (lane == 0) wc[cc][wid] = __popc(b);
    if (c == cc) mine = b;
  }
  __syncthreads();
  // exclusive scan of the per-warp counts of every class (NC warps work)
  if (wid < NC) {
    uint32_t x = wc[wid][lane];
    uint32_t incl = warp_inclusive(x, lane);
    wc[wid][lane] = incl - x;
  }
  __syncthreads();
  if (c >= 0) {
    const uint32_t lt = mine & ((1u << lane) - 1u);
    const uint32_t pos = offsets[c * nblocks + blockIdx.x] + wc[c][wid] + __popc(lt);
    out[pos] = val(i);
  }
}

template <int NC, class ClassFn, class ValueFn>
cudaError_t partition_impl(uint32_t n, ClassFn fn, ValueFn val, uint32_t* out,
                           uint32_t* cls_count, uint32_t* tmp, ScanScratch& s,
                           cudaStream_t st) {
  const uint32_t nb = (n + kPartThreads - 1) / kPartThreads;
  if (nb == 0) {
    cudaError_t e = cudaMemsetAsync(cls_count, 0, NC * sizeof(uint32_t), st);
    return e;
  }
  uint32_t* counts = tmp;             // NC * nb
  uint32_t* grand = tmp + NC * nb;    // 1
  (count_launches(1), part_count_kernel<NC, ClassFn><<<nb, kPartThreads, 0, st>>>(n, fn, counts, nb));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  e = exclusive_scan_u32(counts, counts, (size_t)NC * nb, grand, s, st);
  if (e != cudaSuccess) return e;
  (count_launches(1), part_scatter_kernel<NC, ClassFn, ValueFn>
                         <<<nb, kPartThreads, 0, st>>>(n, fn, val, counts, nb, out, grand,
                                                       cls_count));
  return cudaGetLastError();
}

struct DegreeClass {
  const uint64_t* off;
  __device__ int operator()(uint32_t v) const {
    return move_class_of_degree(off[v + 1] - off[v]);
  }
};
struct Identity {
  __device__ uint32_t operator()(uint32_t i) const { return i; }
};
struct SizeClass4 {
  const uint64_t* sizes;
  const uint32_t* live;  // items i >= *live belong to no class
  uint64_t lim0, lim1, lim2;
  __device__ int operator()(uint32_t i) const {
    if (i >= *live) return -1;
    uint64_t s = sizes[i];
    return s <= lim0 ? 0 : (s <= lim1 ? 1 : (s <= lim2 ? 2 : 3));
  }
};

}  // namespace

size_t scan_scratch_bytes(size_t cap) {
  size_t elems = 0, n = cap;
  do {
    n = tiles_of(n);
    elems += n + 1;
  } while (n > 1);
  return (elems + 64) * sizeof(uint64_t);
}

cudaError_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, size_t n,
                               uint32_t* total, ScanScratch& s,
                               cudaStream_t st) {
  return scan_rec<uint32_t>(in, out, n, total, (uint32_t*)s.buf,
                            s.bytes / sizeof(uint32_t), st);
}

cudaError_t exclusive_scan_u64(const uint64_t* in, uint64_t* out, size_t n,
                               uint64_t* total, ScanScratch& s,
                               cudaStream_t st) {
  return scan_rec<uint64_t>(in, out, n, total, (uint64_t*)s.buf,
                            s.bytes / sizeof(uint64_t), st);
}

size_t partition_tmp_words(size_t n) {
  return (size_t)kClasses * ((n + kPartThreads - 1) / kPartThreads) + 16;
}

cudaError_t partition_by_degree(const uint64_t* off, uint32_t n,
                                uint32_t* order, uint32_t* cls_count,
                                uint32_t* tmp, ScanScratch& s,
                                cudaStream_t st) {
  return partition_impl<kClasses>(n, DegreeClass{off}, Identity{}, order,
                                  cls_count, tmp, s, st);
}

cudaError_t partition_by_size4(const uint64_t* sizes, uint32_t n_upper,
                               const uint32_t* d_live, uint64_t lim0,
                               uint64_t lim1, uint64_t lim2, uint32_t* out,
                               uint32_t* cls_count, uint32_t* tmp,
                               ScanScratch& s, cudaStream_t st) {
  return partition_impl<4>(n_upper, SizeClass4{sizes, d_live, lim0, lim1, lim2},
                           Identity{}, out, cls_count, tmp, s, st);
}

}  // namespace lvb
