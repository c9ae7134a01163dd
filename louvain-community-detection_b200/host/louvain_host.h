// louvain_host.h -- C++ host API with the reference's names and argument
// meanings (utils.cuh:47-76, modularity.cuh:6, aggregation.cuh:6), built
// on the C ABI in include/louvain_b200.h.
//
// Differences from the reference, all in error handling: functions throw
// lvb_host::Error (with the C ABI status) instead of calling exit(), and
// the CLI turns that into the reference's message and exit code.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "louvain_b200.h"

namespace lvb_host {

struct Error : std::runtime_error {
  lv_status status;
  Error(lv_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

// Host graph + device state; stands for the reference's Graph/CommAggr
// pair (utils.cuh:15-45).  Fields mirror the ones the reference reads.
struct Graph {
  lv_graph* host = nullptr;
  lv_engine* dev = nullptr;
  size_t vert_sz = 0;   // current level's vertex count
  size_t edges_sz = 0;  // current level's stored entries
  size_t init_sz = 0;   // input vertex count
  unsigned int max_deg = 0;
  lv_rule rule = LV_RULE_PY;
  std::string path;  // --gpu-csr: the file the engine parses itself
};

// parseGraph (utils.cu:168-229): Matrix Market file -> host CSR.
void parseGraph(Graph& graph, const char* filename);
// This build's --cache: parseGraph keeps a binary CSR beside the file.
void setCsrCache(bool on);
// This build's --gpu-csr: parseGraph only checks the file; initDevGraph
// parses it on the host and builds the CSR on the device
// (lv_engine_load_mtx).
void setDeviceCsr(bool on);

// initDevGraph + copyToDevice + initCommAggr + setInitComm
// (utils.cu:66-108): create the engine and upload the graph.
void initDevGraph(Graph& dev_graph, const Graph& host_graph, const lv_config* cfg);

// modularityOptimization (modularity.cu:438-520): one phase of local
// moving.  Returns false when the algorithm ends, after printing the final
// modularity on stdout exactly as the reference does (modularity.cu:504).
bool modularityOptimization(Graph& dev_graph, float threshold);

// aggregation (aggregation.cu:387-462): contract communities in place.
void aggregation(Graph& dev_graph);

// printCommunities (utils.cu:270-293): community count, then one line per
// community "k v1 v2 ... " with 1-based vertex ids.
void printCommunities(Graph& dev_graph);

// parseArgs (utils.cu:231-267): -f file -g min_gain [-v]; this build adds
// --rule py|cuda, --gain fp32|fp64, --timing (per-level times on stderr),
// --cache and --gpu-csr.
void parseArgs(int argc, char** argv, float& threshold, bool& verbose,
               char*& filename, lv_rule& rule, bool& timing, lv_gain& gain);

// deleteDevGraph / deleteHostGraph (utils.cu:30-64).
void deleteDevGraph(Graph& dev_graph);
void deleteHostGraph(Graph& host_graph);

// Per-level timings of the run so far.
std::vector<lv_level_info> levelInfo(Graph& dev_graph);

}  // namespace lvb_host
