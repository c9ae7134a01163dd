// lv_graph.h -- host CSR graph behind the opaque lv_graph handle.
#pragma once

#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <new>
#include <vector>

#include <cuda_runtime_api.h>

// Host buffers of a graph: page-locked when a CUDA device is present and the
// buffer is at least 1 MiB (its upload then runs at full DMA speed without a
// staging copy, and stays asynchronous), ordinary memory otherwise (no
// device, small buffers, or page-locking refused).  A 64-byte header records
// which kind a block is.
template <class T>
struct HostBufAlloc {
  using value_type = T;
  static constexpr size_t kHeader = 64;
  static constexpr size_t kPinMin = 1u << 20;
  HostBufAlloc() = default;
  template <class U>
  HostBufAlloc(const HostBufAlloc<U>&) {}
  static std::atomic<int>& pin_state() {  // 0 unknown / usable, -1 unavailable
    static std::atomic<int> s{0};
    return s;
  }
  T* allocate(size_t n) {
    const size_t bytes = n * sizeof(T) + kHeader;
    unsigned char* base = nullptr;
    bool pinned = false;
    if (n * sizeof(T) >= kPinMin && pin_state().load() == 0) {
      void* p = nullptr;
      if (cudaHostAlloc(&p, bytes, cudaHostAllocPortable) == cudaSuccess) {
        base = static_cast<unsigned char*>(p);
        pinned = true;
      } else {
        cudaGetLastError();
        pin_state().store(-1);
      }
    }
    if (!base) {
      base = static_cast<unsigned char*>(std::malloc(bytes));
      if (!base) throw std::bad_alloc();
    }
    base[0] = pinned ? 1 : 0;
    return reinterpret_cast<T*>(base + kHeader);
  }
  void deallocate(T* p, size_t) noexcept {
    if (!p) return;
    unsigned char* base = reinterpret_cast<unsigned char*>(p) - kHeader;
    if (base[0]) cudaFreeHost(base);
    else std::free(base);
  }
  template <class U>
  bool operator==(const HostBufAlloc<U>&) const { return true; }
  template <class U>
  bool operator!=(const HostBufAlloc<U>&) const { return false; }
};

template <class T>
using HostVec = std::vector<T, HostBufAlloc<T>>;

struct lv_graph {
  uint32_t n = 0;
  uint64_t nnz = 0;
  uint32_t max_deg = 0;
  HostVec<uint64_t> off;  // n + 1
  HostVec<uint32_t> col;  // nnz
  HostVec<float> w;       // nnz
};
