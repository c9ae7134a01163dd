// main.cpp -- CLI with the reference's interface (main.cu:5-70):
//   louvain -f <file.mtx> -g <min_gain> [-v] [--rule py|cuda] [--gain fp32|fp64]
//           [--timing] [--cache]
// stdout: final modularity (6 significant digits), then "alg_ms total_ms";
// with -v the community count and one "k v1 v2 ..." line per community.
// --timing adds a per-level table on stderr (stdout stays as the
// reference's).
#include <chrono>
#include <cstdio>
#include <iostream>

#include "louvain_host.h"

using namespace lvb_host;

int main(int argc, char** argv) {
  char* filename = nullptr;
  float threshold = 0.0f;
  bool verbose = false, timing = false;
  lv_rule rule = LV_RULE_PY;
  lv_gain gain = LV_GAIN_FP32;
  parseArgs(argc, argv, threshold, verbose, filename, rule, timing, gain);

  Graph host_graph, dev_graph;
  try {
    parseGraph(host_graph, filename);
  } catch (const Error& e) {
    if (e.status == LV_ERR_IO) {
      std::cout << "Error opening file" << std::endl;  // utils.cu:172
    } else {
      std::cout << e.what() << std::endl;
    }
    return 1;
  }
  try {
    lv_config cfg;
    lv_config_default(&cfg);
    cfg.rule = rule;
    cfg.gain = gain;
    // "copy" region (main.cu:19-35): engine set-up and upload
    auto c0 = std::chrono::steady_clock::now();
    initDevGraph(dev_graph, host_graph, &cfg);
    auto c1 = std::chrono::steady_clock::now();
    const float copy_ms =
        std::chrono::duration<float, std::milli>(c1 - c0).count();
    // "alg" region (main.cu:37-56)
    auto a0 = std::chrono::steady_clock::now();
    for (;;) {
      const size_t before = dev_graph.vert_sz;
      if (!modularityOptimization(dev_graph, threshold)) break;
      aggregation(dev_graph);
      if (dev_graph.vert_sz == before) {
        // nothing merged (threshold <= 0): report the partition and stop
        uint32_t count = 0;
        lv_get_levels(dev_graph.dev, nullptr, 0, &count);
        std::vector<lv_level_info> lv = levelInfo(dev_graph);
        std::cout << static_cast<float>(lv.empty() ? 0.0 : lv.back().q_end) << std::endl;
        break;
      }
    }
    auto a1 = std::chrono::steady_clock::now();
    const float alg_ms = std::chrono::duration<float, std::milli>(a1 - a0).count();
    std::cout << alg_ms << " " << alg_ms + copy_ms << std::endl;
    if (timing) {
      std::vector<lv_level_info> lv = levelInfo(dev_graph);
      std::fprintf(stderr, "level  vertices      entries  passes  q_start     q_end       move_ms  aggr_ms\n");
      for (size_t i = 0; i < lv.size(); i++) {
        std::fprintf(stderr, "%5zu %9u %12llu %7u  %.8f  %.8f %8.3f %8.3f\n", i,
                     lv[i].n_vertices, (unsigned long long)lv[i].n_entries, lv[i].passes,
                     lv[i].q_start, lv[i].q_end, lv[i].move_ms, lv[i].aggregate_ms);
      }
    }
    if (verbose) printCommunities(dev_graph);
  } catch (const Error& e) {
    std::cout << e.what() << std::endl;
    deleteDevGraph(dev_graph);
    deleteHostGraph(host_graph);
    return 1;
  }
  deleteDevGraph(dev_graph);
  deleteHostGraph(host_graph);
  return 0;
}
