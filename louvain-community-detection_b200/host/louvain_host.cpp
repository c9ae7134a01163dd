// louvain_host.cpp -- the reference-named C++ host API over the C ABI.
#include "louvain_host.h"

#include <getopt.h>
#include <sys/stat.h>

#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <iterator>
#include <string>

namespace lvb_host {

static void check(lv_status s) {
  if (s != LV_OK) throw Error(s, lv_last_error());
}

static bool g_use_cache = false;
void setCsrCache(bool on) { g_use_cache = on; }
static bool g_device_csr = false;
void setDeviceCsr(bool on) { g_device_csr = on; }

// With the cache on, `<file>.lvbcsr` (a binary CSR newer than the file)
// replaces the text parse, and is written after a parse.
void parseGraph(Graph& graph, const char* filename) {
  if (g_device_csr) {  // the engine parses and builds the CSR on the device
    FILE* f = fopen(filename, "rb");
    if (!f) throw Error(LV_ERR_IO, "Error opening file");
    fclose(f);
    graph.path = filename;
    return;
  }
  lv_graph* g = nullptr;
  const std::string cache = std::string(filename) + ".lvbcsr";
  struct stat sm {}, sc {};
  const bool fresh = g_use_cache && stat(filename, &sm) == 0 && stat(cache.c_str(), &sc) == 0 &&
                     sc.st_mtime >= sm.st_mtime;
  if (!fresh || lv_graph_load(cache.c_str(), &g) != LV_OK) {
    g = nullptr;
    check(lv_graph_load_mtx(filename, &g));
    if (g_use_cache) lv_graph_save(g, cache.c_str());  // best effort
  }
  graph.host = g;
  uint32_t n = 0, md = 0;
  uint64_t e = 0;
  check(lv_graph_view(g, &n, &e, nullptr, nullptr, nullptr, &md));
  graph.vert_sz = n;
  graph.init_sz = n;
  graph.edges_sz = e;
  graph.max_deg = md;
}

void initDevGraph(Graph& dev_graph, const Graph& host_graph, const lv_config* cfg) {
  lv_engine* e = nullptr;
  check(lv_engine_create(cfg, &e));
  dev_graph.dev = e;
  dev_graph.rule = cfg ? cfg->rule : LV_RULE_PY;
  lv_status s = host_graph.host ? lv_engine_load(e, host_graph.host)
                                : lv_engine_load_mtx(e, host_graph.path.c_str());
  if (s != LV_OK) {
    lv_engine_destroy(e);
    dev_graph.dev = nullptr;
    check(s);
  }
  if (host_graph.host) {
    dev_graph.vert_sz = host_graph.vert_sz;
    dev_graph.init_sz = host_graph.init_sz;
    dev_graph.edges_sz = host_graph.edges_sz;
    dev_graph.max_deg = host_graph.max_deg;
  } else {
    uint32_t n = 0;
    uint64_t ne = 0;
    check(lv_get_level_size(e, &n, &ne));
    dev_graph.vert_sz = dev_graph.init_sz = n;
    dev_graph.edges_sz = ne;
  }
}

bool modularityOptimization(Graph& dev_graph, float threshold) {
  int more = 0;
  double q = 0.0;
  check(lv_phase_move(dev_graph.dev, threshold, &more, &q));
  if (!more) {
    // modularity.cu:504 prints the FP32 value with default stream format
    std::cout << static_cast<float>(q) << std::endl;
  }
  return more != 0;
}

void aggregation(Graph& dev_graph) {
  check(lv_phase_aggregate(dev_graph.dev));
  uint32_t n = 0;
  uint64_t e = 0;
  check(lv_get_level_size(dev_graph.dev, &n, &e));
  dev_graph.vert_sz = n;
  dev_graph.edges_sz = e;
}

// The vertices grouped by community on the device (lv_get_communities:
// a stable sort by community, so vertex ids stay ascending inside a
// community, as the reference's push_back order leaves them; one copy to
// the host), written through one buffer.
void printCommunities(Graph& dev_graph) {
  const size_t n0 = dev_graph.init_sz;
  uint32_t c = 0;
  check(lv_get_communities(dev_graph.dev, nullptr, 0, &c));
  std::vector<uint32_t> grouped((size_t)c + 1 + n0);
  check(lv_get_communities(dev_graph.dev, grouped.data(), grouped.size(), &c));
  const size_t nc = c;
  const uint32_t* start = grouped.data();
  const uint32_t* members = grouped.data() + nc + 1;
  std::string out;
  out.reserve(16 * (n0 + nc) + 32);
  char num[24];
  auto put = [&](uint64_t v) {
    int k = 0;
    do {
      num[k++] = (char)('0' + v % 10);
      v /= 10;
    } while (v);
    while (k) out.push_back(num[--k]);
  };
  put(nc);
  out.push_back('\n');
  uint64_t comm_n = 1;
  for (size_t c = 0; c < nc; c++) {
    if (start[c] == start[c + 1]) continue;
    put(comm_n++);
    out.push_back(' ');
    for (uint64_t k = start[c]; k < start[c + 1]; k++) {
      put((uint64_t)members[k] + 1);  // 1-based, utils.cu:287
      out.push_back(' ');
    }
    out.push_back('\n');
  }
  std::cout.write(out.data(), (std::streamsize)out.size());
  std::cout.flush();
}

void parseArgs(int argc, char** argv, float& threshold, bool& verbose,
               char*& filename, lv_rule& rule, bool& timing, lv_gain& gain) {
  static const struct option longopts[] = {
      {"rule", required_argument, nullptr, 'r'},
      {"gain", required_argument, nullptr, 'p'},
      {"timing", no_argument, nullptr, 't'},
      {"cache", no_argument, nullptr, 'c'},
      {"gpu-csr", no_argument, nullptr, 'd'},
      {nullptr, 0, nullptr, 0}};
  const char* usage = "Usage: ./gpulouvain -f mtx-matrix-file -g min-gain [-v]";
  bool fopt = false, gopt = false;
  int c;
  while ((c = getopt_long(argc, argv, "f:g:v", longopts, nullptr)) != -1) {
    switch (c) {
      case 'f':
        filename = optarg;
        fopt = true;
        break;
      case 'g':
        try {
          threshold = std::stof(std::string(optarg));
        } catch (const std::invalid_argument& ia) {
          std::cout << "-g option invalid argument: " << ia.what() << std::endl;
          exit(1);
        } catch (const std::out_of_range& oor) {
          std::cout << "-g option error out of range: " << oor.what() << std::endl;
          exit(1);
        }
        gopt = true;
        break;
      case 'v':
        verbose = true;
        break;
      case 'r':
        if (std::string(optarg) == "py") {
          rule = LV_RULE_PY;
        } else if (std::string(optarg) == "cuda") {
          rule = LV_RULE_CUDA;
        } else {
          std::cout << "--rule must be py or cuda" << std::endl;
          exit(1);
        }
        break;
      case 'p':
        if (std::string(optarg) == "fp32") {
          gain = LV_GAIN_FP32;
        } else if (std::string(optarg) == "fp64") {
          gain = LV_GAIN_FP64;
        } else {
          std::cout << "--gain must be fp32 or fp64" << std::endl;
          exit(1);
        }
        break;
      case 't':
        timing = true;
        break;
      case 'c':
        setCsrCache(true);
        break;
      case 'd':
        setDeviceCsr(true);
        break;
      case '?':
        std::cout << usage << std::endl;
        exit(1);
      default:
        std::cout << "?? arg_parser error ??" << std::endl;
    }
  }
  if (!fopt || !gopt) {
    std::cout << usage << std::endl;
    exit(1);
  }
}

void deleteDevGraph(Graph& dev_graph) {
  lv_engine_destroy(dev_graph.dev);
  dev_graph.dev = nullptr;
}

void deleteHostGraph(Graph& host_graph) {
  lv_graph_destroy(host_graph.host);
  host_graph.host = nullptr;
}

std::vector<lv_level_info> levelInfo(Graph& dev_graph) {
  uint32_t count = 0;
  check(lv_get_levels(dev_graph.dev, nullptr, 0, &count));
  std::vector<lv_level_info> v(count);
  check(lv_get_levels(dev_graph.dev, v.data(), count, &count));
  return v;
}

}  // namespace lvb_host
