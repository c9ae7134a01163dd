// noalloc.cu -- FP64 modularity of a partition without any allocation.
//
// Some callers cannot allocate device memory on the call path: serving
// loops with a latency budget that must not stall on the allocator (and
// cannot afford the device-wide synchronisation of a cudaFree), and
// processes whose device memory is owned by another allocator (a
// framework's caching allocator, a fixed budget carved out at start-up)
// and so cannot be grown behind that allocator's back.  For them,
// lv_modularity_noalloc computes what lv_modularity_fp64 computes, with
// its scratch (one FP64 total per community plus four accumulators) in a
// file-scope __device__ array of fixed size instead of engine buffers.
//
// Limits and sharing:
//   * at most kNoAllocMaxVertices vertices (the array holds one total per
//     community id and ids are < n); larger inputs return LV_ERR_LIMIT;
//   * the array exists once per device that loads the library and stays
//     allocated until the process exits (kNoAllocMaxVertices * 8 bytes,
//     8 MiB, plus a few accumulators);
//   * every call uses the same array and clears it first; calls whose work
//     overlaps on the GPU (other host threads, or other streams) race on it;
//   * every call waits for its stream to finish the work (it reads back
//     whether any community id was invalid);
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture begins.
#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/louvain_b200.h"
#include "lv_internal.h"

void lvb_set_error(const std::string& msg);

namespace lvb {
namespace {

constexpr uint32_t kNoAllocMaxVertices = 1u << 20;
constexpr uint32_t kAcc = kNoAllocMaxVertices;  // intra, asq, total, bad ids
constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxVertices + 32];

std::mutex g_setup_mu;
double* g_scratch_ptr[kMaxDevices] = {};

__global__ void na_clear_kernel(double* s, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x)
    s[i] = 0.0;
  if (blockIdx.x == 0 && threadIdx.x < 4) s[kAcc + threadIdx.x] = 0.0;
}

// community totals a_c = sum of the members' weighted degrees
__global__ void na_totals_kernel(uint32_t n, const uint64_t* off, const float* w,
                                 const uint32_t* part, double* s) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += gridDim.x * blockDim.x) {
    const uint32_t c = part[v];
    if (c >= n) {  // invalid id: record it, skip the access
      atomicAdd(&s[kAcc + 3], 1.0);
      continue;
    }
    double k = 0.0;
    for (uint64_t j = off[v]; j < off[v + 1]; j++) k += (double)w[j];
    atomicAdd(&s[c], k);
  }
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// intra-community weight, squared totals, total weight
__global__ void __launch_bounds__(256)
    na_sums_kernel(uint32_t n, const uint64_t* off, const uint32_t* col,
                   const float* w, const uint32_t* part, double* s) {
  __shared__ double red[3][8];
  double intra = 0.0, asq = 0.0, all = 0.0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += gridDim.x * blockDim.x) {
    const uint32_t p = part[v];
    for (uint64_t j = off[v]; j < off[v + 1]; j++) {
      const double x = (double)w[j];
      all += x;
      const uint32_t u = col[j];
      if (u < n && part[u] == p) intra += x;
    }
    const double a = s[v];
    asq += a * a;
  }
  intra = warp_sum(intra);
  asq = warp_sum(asq);
  all = warp_sum(all);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][wid] = intra;
    red[1][wid] = asq;
    red[2][wid] = all;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0.0;
    for (int i = 0; i < 8; i++) t += red[threadIdx.x][i];
    atomicAdd(&s[kAcc + threadIdx.x], t);
  }
}

// Q, or NaN when some community id was out of range (the sums then miss
// those vertices, so no Q is meaningful).
__global__ void na_final_kernel(const double* s, double* q) {
  if (s[kAcc + 3] != 0.0) {
    *q = __longlong_as_double(0x7ff8000000000000ll);
    return;
  }
  const double m = s[kAcc + 2] / 2.0;
  *q = (m > 0.0) ? s[kAcc + 0] / (2.0 * m) - s[kAcc + 1] / (4.0 * m * m) : 0.0;
}

// Looks up the scratch array's device address for the current device once.
lv_status scratch_for_current_device(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    lvb_set_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    return LV_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    lvb_set_error("device ordinal beyond the supported range");
    return LV_ERR_LIMIT;
  }
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      lvb_set_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return LV_ERR_CUDA;
    }
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[dev];
  return LV_OK;
}

}  // namespace
}  // namespace lvb

using namespace lvb;

extern "C" lv_status lv_modularity_noalloc(uint32_t n_vertices, const uint64_t* d_offsets,
                                           const uint32_t* d_cols, const float* d_weights,
                                           const uint32_t* d_partition, double* d_q,
                                           double* q_host, void* stream) {
  if (!d_offsets || !d_partition || !d_q) {
    lvb_set_error("NULL device pointer");
    return LV_ERR_ARG;
  }
  if (n_vertices > 0 && (!d_cols || !d_weights)) {
    lvb_set_error("lv_modularity_noalloc: NULL columns or weights for a non-empty graph");
    return LV_ERR_ARG;
  }
  if (n_vertices > kNoAllocMaxVertices) {
    lvb_set_error("lv_modularity_noalloc: at most " + std::to_string(kNoAllocMaxVertices) +
                  " vertices (its fixed scratch holds one total per community)");
    return LV_ERR_LIMIT;
  }
  double* s = nullptr;
  lv_status st = scratch_for_current_device(&s);
  if (st != LV_OK) return st;
  cudaStream_t cs = static_cast<cudaStream_t>(stream);
  const uint32_t n = n_vertices;
  const unsigned g = n ? std::min<unsigned>((n + 255) / 256, 148 * 8) : 1;
  (count_launches(1), na_clear_kernel<<<g, 256, 0, cs>>>(s, n));
  if (n) {
    (count_launches(1), na_totals_kernel<<<g, 256, 0, cs>>>(n, d_offsets, d_weights,
                                                           d_partition, s));
    (count_launches(1), na_sums_kernel<<<g, 256, 0, cs>>>(n, d_offsets, d_cols, d_weights,
                                                         d_partition, s));
  }
  (count_launches(1), na_final_kernel<<<1, 1, 0, cs>>>(s, d_q));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    lvb_set_error(std::string("lv_modularity_noalloc launch: ") + cudaGetErrorString(e));
    return LV_ERR_CUDA;
  }
  double bad = 0.0;
  e = cudaMemcpyAsync(&bad, s + kAcc + 3, sizeof(double), cudaMemcpyDeviceToHost, cs);
  if (e == cudaSuccess && q_host)
    e = cudaMemcpyAsync(q_host, d_q, sizeof(double), cudaMemcpyDeviceToHost, cs);
  if (e == cudaSuccess) e = cudaStreamSynchronize(cs);
  if (e != cudaSuccess) {
    lvb_set_error(std::string("lv_modularity_noalloc: ") + cudaGetErrorString(e));
    return LV_ERR_CUDA;
  }
  if (bad != 0.0) {
    lvb_set_error("lv_modularity_noalloc: a community id is >= the vertex count");
    return LV_ERR_ARG;
  }
  return LV_OK;
}
