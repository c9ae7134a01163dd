// lv_graph.h -- host CSR graph behind the opaque lv_graph handle.
#pragma once

#include <cstdint>
#include <vector>

struct lv_graph {
  uint32_t n = 0;
  uint64_t nnz = 0;
  uint32_t max_deg = 0;
  std::vector<uint64_t> off;  // n + 1
  std::vector<uint32_t> col;  // nnz
  std::vector<float> w;       // nnz
};
