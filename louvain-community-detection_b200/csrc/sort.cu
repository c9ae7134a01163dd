// sort.cu -- stable device radix sort, and the two ingest / output steps
// built on it: the CSR of an edge list and the community listing.
//
// Reference counterparts (upicine/louvain-community-detection):
//   parseGraph's CSR construction ........ utils.cu:168-229 (host, one
//                                          vector per row, file order)
//   printCommunities's grouping ........... utils.cu:270-293 (host, one
//                                          scan over init_comm per community)
//
// Radix sort: least-significant digit first, 8-bit digits, one pass per
// digit of the key bits in use.  A pass is three launches over tiles of
// 4096 keys: a per-tile digit histogram (stored digit-major, so one
// exclusive scan of the whole table gives every (digit, tile) its output
// offset), the scan, and a scatter in which each warp ranks its 512 keys
// round by round (equal digits of a round found with __match_any_sync), so
// the order of equal keys is kept: the sort is stable.
#include <algorithm>

#include "lv_internal.h"

namespace lvb {
namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;                           // keys per thread
constexpr uint32_t kSortTile = kSortThreads * kSortItems;  // 4096
constexpr uint32_t kWarpKeys = kSortTile / kSortWarps;     // 512 per warp
constexpr int kRadix = 256;

template <typename K>
__device__ __forceinline__ uint32_t digit_of(K k, int shift) {
  return (uint32_t)(k >> shift) & (kRadix - 1);
}

// counts[d * tiles + t] = keys of tile t with digit d.
template <typename K>
__global__ void __launch_bounds__(kSortThreads)
    radix_hist_kernel(const K* __restrict__ keys, uint64_t n, int shift, uint32_t tiles,
                      uint32_t* __restrict__ counts) {
  __shared__ uint32_t h[kRadix];
  for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    for (int d = threadIdx.x; d < kRadix; d += kSortThreads) h[d] = 0u;
    __syncthreads();
    const uint64_t base = (uint64_t)t * kSortTile;
#pragma unroll 4
    for (int i = 0; i < kSortItems; i++) {
      const uint64_t j = base + (uint64_t)i * kSortThreads + threadIdx.x;
      if (j < n) atomicAdd(&h[digit_of(keys[j], shift)], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += kSortThreads)
      counts[(uint64_t)d * tiles + t] = h[d];
    __syncthreads();
  }
}

// Stable scatter of one tile: warp w owns keys [w*512, (w+1)*512) of the
// tile, in order; offsets holds the scanned counts.
template <typename K>
__global__ void __launch_bounds__(kSortThreads)
    radix_scatter_kernel(const K* __restrict__ keys, const uint32_t* __restrict__ vals,
                         uint64_t n, int shift, uint32_t tiles,
                         const uint32_t* __restrict__ offsets, K* __restrict__ keys_out,
                         uint32_t* __restrict__ vals_out) {
  __shared__ uint32_t wbase[kSortWarps][kRadix];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    for (int i = threadIdx.x; i < kSortWarps * kRadix; i += kSortThreads)
      (&wbase[0][0])[i] = 0u;
    __syncthreads();
    const uint64_t wb = (uint64_t)t * kSortTile + (uint64_t)wid * kWarpKeys;
    // this warp's digit counts
    for (uint32_t r = 0; r < kWarpKeys; r += 32) {
      const uint64_t j = wb + r + lane;
      if (j < n) atomicAdd(&wbase[wid][digit_of(keys[j], shift)], 1u);
    }
    __syncthreads();
    // per digit: the tile's offset, then the warps in order
    for (int d = threadIdx.x; d < kRadix; d += kSortThreads) {
      uint32_t run = offsets[(uint64_t)d * tiles + t];
      for (int w = 0; w < kSortWarps; w++) {
        const uint32_t c = wbase[w][d];
        wbase[w][d] = run;
        run += c;
      }
    }
    __syncthreads();
    for (uint32_t r = 0; r < kWarpKeys; r += 32) {
      const uint64_t j = wb + r + lane;
      const bool valid = j < n;
      K k = 0;
      uint32_t v = 0, d = 0x100u + lane;  // distinct sentinels for idle lanes
      if (valid) {
        k = keys[j];
        v = vals[j];
        d = digit_of(k, shift);
      }
      const unsigned peers = __match_any_sync(0xffffffffu, d);
      const uint32_t rank = __popc(peers & lt);
      const int leader = __ffs(peers) - 1;
      uint32_t base = 0;
      if (valid) base = wbase[wid][d];
      __syncwarp();
      if (valid) {
        const uint32_t pos = base + rank;
        keys_out[pos] = k;
        vals_out[pos] = v;
        if (lane == leader) wbase[wid][d] = base + __popc(peers);
      }
      __syncwarp();
    }
    __syncthreads();
  }
}

unsigned sort_grid(uint32_t tiles) {
  const unsigned cap = sm_count_cached() * 8;
  return tiles < cap ? (tiles ? tiles : 1u) : cap;
}

// ---------------------------------------------------------------------------
// CSR of an edge list
// ---------------------------------------------------------------------------
// Directed entries in the order the reference reader appends them
// (utils.cu:302-313): edge e gives entry 2e in row src[e] and, unless it is
// a self-loop, entry 2e+1 in row dst[e]; a self-loop's second entry gets the
// key n and sorts after every row.
__global__ void expand_edges_kernel(const uint32_t* __restrict__ src,
                                    const uint32_t* __restrict__ dst, uint64_t m, uint32_t n,
                                    uint32_t* __restrict__ keys, uint32_t* __restrict__ vals,
                                    uint32_t* __restrict__ bad) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t a = src[e], b = dst[e];
    if (a >= n || b >= n) atomicExch(bad, 1u);
    keys[2 * e] = a < n ? a : n;
    vals[2 * e] = (uint32_t)(2 * e);
    keys[2 * e + 1] = (a != b && b < n) ? b : n;
    vals[2 * e + 1] = (uint32_t)(2 * e + 1);
  }
}

// off[v] = first position whose key is >= v, for v in [0, n]: position j
// writes the rows between the previous key and its own.
__global__ void bounds_from_sorted_kernel(const uint32_t* __restrict__ keys, uint64_t total,
                                          uint32_t n, uint64_t* __restrict__ off) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j <= total;
       j += (uint64_t)gridDim.x * blockDim.x) {
    const int64_t prev = j ? (int64_t)keys[j - 1] : -1;
    const uint32_t cur = j < total ? keys[j] : n;
    for (int64_t v = prev + 1; v <= (int64_t)cur && v <= (int64_t)n; v++) off[v] = j;
  }
}

// The entries' columns and weights from the sorted entry ids (|w| as
// utils.cu:295; weight 1 without a weight array).
__global__ void gather_entries_kernel(const uint32_t* __restrict__ ids, const uint64_t* off_n,
                                      const uint32_t* __restrict__ src,
                                      const uint32_t* __restrict__ dst,
                                      const float* __restrict__ w, uint32_t* __restrict__ col,
                                      float* __restrict__ wout) {
  const uint64_t nnz = *off_n;
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < nnz;
       j += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t id = ids[j];
    const uint64_t e = id >> 1;
    col[j] = (id & 1u) ? src[e] : dst[e];
    wout[j] = w ? fabsf(w[e]) : 1.0f;
  }
}

__global__ void narrow_u64_kernel(const uint64_t* __restrict__ in, uint64_t n,
                                  uint32_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = (uint32_t)in[i];
}

__global__ void iota_u32_kernel(uint32_t* a, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    a[i] = (uint32_t)i;
}

int bits_for(uint64_t max_key) {
  int b = 0;
  while (b < 64 && (max_key >> b)) b++;
  return b;
}

template <typename T>
cudaError_t salloc(T** p, size_t count, cudaStream_t st) {
  return cudaMallocAsync((void**)p, std::max<size_t>(count, 1) * sizeof(T), st);
}

}  // namespace

size_t radix_sort_scratch_words(uint64_t n) {
  const uint64_t tiles = (n + kSortTile - 1) / kSortTile;
  return (size_t)tiles * kRadix + 64;
}

template <typename K>
cudaError_t radix_sort_pairs(K* keys, uint32_t* vals, K* keys_alt, uint32_t* vals_alt,
                             uint64_t n, int key_bits, uint32_t* counts, ScanScratch& S,
                             cudaStream_t st, bool* result_in_alt) {
  *result_in_alt = false;
  if (n <= 1 || key_bits <= 0) return cudaSuccess;
  const uint32_t tiles = (uint32_t)((n + kSortTile - 1) / kSortTile);
  const unsigned grid = sort_grid(tiles);
  K* kin = keys;
  uint32_t* vin = vals;
  K* kout = keys_alt;
  uint32_t* vout = vals_alt;
  for (int shift = 0; shift < key_bits; shift += 8) {
    (count_launches(1), radix_hist_kernel<K><<<grid, kSortThreads, 0, st>>>(kin, n, shift, tiles,
                                                                              counts));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = exclusive_scan_u32(counts, counts, (size_t)tiles * kRadix, nullptr, S, st);
    if (e != cudaSuccess) return e;
    (count_launches(1), radix_scatter_kernel<K><<<grid, kSortThreads, 0, st>>>(
                            kin, vin, n, shift, tiles, counts, kout, vout));
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    std::swap(kin, kout);
    std::swap(vin, vout);
    *result_in_alt = !*result_in_alt;
  }
  return cudaSuccess;
}

template cudaError_t radix_sort_pairs<uint32_t>(uint32_t*, uint32_t*, uint32_t*, uint32_t*,
                                                uint64_t, int, uint32_t*, ScanScratch&,
                                                cudaStream_t, bool*);
template cudaError_t radix_sort_pairs<uint64_t>(uint64_t*, uint32_t*, uint64_t*, uint32_t*,
                                                uint64_t, int, uint32_t*, ScanScratch&,
                                                cudaStream_t, bool*);

cudaError_t csr_from_edges_device(uint32_t n, uint64_t m, const uint32_t* src,
                                  const uint32_t* dst, const float* w, uint64_t* off,
                                  uint32_t* col, float* wout, uint64_t* nnz_host,
                                  uint32_t* bad_host, cudaStream_t st) {
  const uint64_t total = 2 * m;
  uint32_t *keys = nullptr, *vals = nullptr, *keys2 = nullptr, *vals2 = nullptr;
  uint32_t *counts = nullptr, *bad = nullptr;
  ScanScratch S;
  cudaError_t e = cudaSuccess;
  const size_t cw = radix_sort_scratch_words(total);
  S.bytes = scan_scratch_bytes(cw);
  if ((e = salloc(&keys, total, st)) != cudaSuccess ||
      (e = salloc(&vals, total, st)) != cudaSuccess ||
      (e = salloc(&keys2, total, st)) != cudaSuccess ||
      (e = salloc(&vals2, total, st)) != cudaSuccess ||
      (e = salloc(&counts, cw, st)) != cudaSuccess ||
      (e = salloc(&bad, 1, st)) != cudaSuccess ||
      (e = cudaMallocAsync(&S.buf, S.bytes, st)) != cudaSuccess) {
    goto done;
  }
  {
    const unsigned g = sort_grid((uint32_t)std::min<uint64_t>((m + 255) / 256, 1u << 30));
    if ((e = cudaMemsetAsync(bad, 0, sizeof(uint32_t), st)) != cudaSuccess) goto done;
    if (m) {
      (count_launches(1), expand_edges_kernel<<<g, 256, 0, st>>>(src, dst, m, n, keys, vals, bad));
      if ((e = cudaGetLastError()) != cudaSuccess) goto done;
    }
    bool alt = false;
    e = radix_sort_pairs<uint32_t>(keys, vals, keys2, vals2, total, bits_for(n), counts, S, st,
                                   &alt);
    if (e != cudaSuccess) goto done;
    const uint32_t* sk = alt ? keys2 : keys;
    const uint32_t* sv = alt ? vals2 : vals;
    const unsigned gb = sort_grid((uint32_t)std::min<uint64_t>((total + 256) / 256, 1u << 30));
    (count_launches(1), bounds_from_sorted_kernel<<<gb, 256, 0, st>>>(sk, total, n, off));
    if ((e = cudaGetLastError()) != cudaSuccess) goto done;
    (count_launches(1), gather_entries_kernel<<<gb, 256, 0, st>>>(sv, off + n, src, dst, w, col,
                                                                   wout));
    if ((e = cudaGetLastError()) != cudaSuccess) goto done;
    if ((e = cudaMemcpyAsync(nnz_host, off + n, sizeof(uint64_t), cudaMemcpyDeviceToHost, st)) !=
        cudaSuccess)
      goto done;
    if ((e = cudaMemcpyAsync(bad_host, bad, sizeof(uint32_t), cudaMemcpyDeviceToHost, st)) !=
        cudaSuccess)
      goto done;
    e = counted_sync(st);
  }
done:
  if (keys) cudaFreeAsync(keys, st);
  if (vals) cudaFreeAsync(vals, st);
  if (keys2) cudaFreeAsync(keys2, st);
  if (vals2) cudaFreeAsync(vals2, st);
  if (counts) cudaFreeAsync(counts, st);
  if (bad) cudaFreeAsync(bad, st);
  if (S.buf) cudaFreeAsync(S.buf, st);
  return e;
}

cudaError_t group_by_community(const uint32_t* part, uint32_t n, uint32_t n_comm,
                               uint32_t* out /* [n_comm + 1 + n] */, cudaStream_t st) {
  uint32_t *keys = nullptr, *vals = nullptr, *keys2 = nullptr, *vals2 = nullptr;
  uint32_t* counts = nullptr;
  uint64_t* off = nullptr;
  ScanScratch S;
  cudaError_t e = cudaSuccess;
  const size_t cw = radix_sort_scratch_words(n);
  S.bytes = scan_scratch_bytes(cw);
  if ((e = salloc(&keys, n, st)) != cudaSuccess || (e = salloc(&vals, n, st)) != cudaSuccess ||
      (e = salloc(&keys2, n, st)) != cudaSuccess ||
      (e = salloc(&vals2, n, st)) != cudaSuccess ||
      (e = salloc(&counts, cw, st)) != cudaSuccess ||
      (e = salloc(&off, (size_t)n_comm + 1, st)) != cudaSuccess ||
      (e = cudaMallocAsync(&S.buf, S.bytes, st)) != cudaSuccess) {
    goto done;
  }
  {
    const unsigned g = sort_grid((uint32_t)std::min<uint64_t>(((uint64_t)n + 255) / 256, 1u << 30));
    if ((e = cudaMemcpyAsync(keys, part, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                             st)) != cudaSuccess)
      goto done;
    (count_launches(1), iota_u32_kernel<<<g, 256, 0, st>>>(vals, n));
    if ((e = cudaGetLastError()) != cudaSuccess) goto done;
    bool alt = false;
    // vertices start in ascending order and the sort is stable: each
    // community's members come out ascending (utils.cu:280-289 prints them
    // so)
    e = radix_sort_pairs<uint32_t>(keys, vals, keys2, vals2, n, bits_for(n_comm ? n_comm - 1 : 0),
                                   counts, S, st, &alt);
    if (e != cudaSuccess) goto done;
    const uint32_t* sk = alt ? keys2 : keys;
    const uint32_t* sv = alt ? vals2 : vals;
    (count_launches(1), bounds_from_sorted_kernel<<<g, 256, 0, st>>>(sk, n, n_comm, off));
    if ((e = cudaGetLastError()) != cudaSuccess) goto done;
    (count_launches(1), narrow_u64_kernel<<<g, 256, 0, st>>>(off, (uint64_t)n_comm + 1, out));
    if ((e = cudaGetLastError()) != cudaSuccess) goto done;
    e = cudaMemcpyAsync(out + n_comm + 1, sv, (size_t)n * sizeof(uint32_t),
                        cudaMemcpyDeviceToDevice, st);
  }
done:
  if (keys) cudaFreeAsync(keys, st);
  if (vals) cudaFreeAsync(vals, st);
  if (keys2) cudaFreeAsync(keys2, st);
  if (vals2) cudaFreeAsync(vals2, st);
  if (counts) cudaFreeAsync(counts, st);
  if (off) cudaFreeAsync(off, st);
  if (S.buf) cudaFreeAsync(S.buf, st);
  return e;
}

}  // namespace lvb
