// graph_io.cpp -- Matrix Market input and host CSR construction.
//
// Semantics of the reference reader (utils.cu:132-229):
//   * lines starting with '%' before the size line are skipped (:137-139);
//   * the size line is `rows cols nnz`; the vertex count is cols (:142);
//   * indices are 0-based if any of the nnz entry lines holds a 0, else
//     1-based (:143-166, :297-300);
//   * the weight is |w| (:295), 1.0 when absent (:289); a line without a
//     weight keeps the previous line's (the stream leaves `weight` as is);
//   * i != j is stored in row i and row j, i == j once (:302-313);
//   * every row keeps file order (:200-227, vector push_back per row).
// Where the reference has undefined behaviour (an index past the size
// line's count, a line without two indices, fewer lines than nnz) this
// reader returns LV_ERR_PARSE instead.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include "../../include/louvain_b200.h"
#include "lv_graph.h"

// Records the calling thread's last error (defined in engine.cu).
void lvb_set_error(const std::string& msg);

namespace {

lv_status io_fail(lv_status s, const std::string& m) {
  lvb_set_error(m);
  return s;
}

bool parse_u64(const char*& p, const char* end, uint64_t* out) {
  while (p < end && (*p == ' ' || *p == '\t' || *p == '\r')) p++;
  if (p >= end || *p < '0' || *p > '9') return false;
  uint64_t v = 0;
  while (p < end && *p >= '0' && *p <= '9') {
    const uint64_t d = (uint64_t)(*p - '0');
    if (v > (UINT64_MAX - d) / 10) return false;
    v = v * 10 + d;
    p++;
  }
  if (p < end && *p != ' ' && *p != '\t' && *p != '\r' && *p != '\n') return false;
  *out = v;
  return true;
}

// returns 1 parsed, 0 no token, -1 malformed
int parse_weight(const char*& p, const char* end, float* out) {
  while (p < end && (*p == ' ' || *p == '\t' || *p == '\r')) p++;
  if (p >= end || *p == '\n') return 0;
  char buf[64];
  size_t len = 0;
  while (p < end && *p != ' ' && *p != '\t' && *p != '\r' && *p != '\n') {
    if (len + 1 < sizeof(buf)) buf[len++] = *p;
    p++;
  }
  buf[len] = '\0';
  char* e = nullptr;
  float v = strtof(buf, &e);
  if (e == buf) return -1;
  *out = v;
  return 1;
}

}  // namespace

// Builds the reference CSR from edge lines (0-based, already validated).
lv_status lvb_graph_build(uint32_t n, uint64_t m, const uint32_t* src,
                          const uint32_t* dst, const float* w, lv_graph** out,
                          std::string* err) {
  lv_graph* g = new (std::nothrow) lv_graph();
  if (!g) return LV_ERR_NOMEM;
  try {
    g->n = n;
    g->off.assign((size_t)n + 1, 0);
    for (uint64_t i = 0; i < m; i++) {
      if (src[i] >= n || dst[i] >= n) {
        if (err) *err = "vertex index exceeds the vertex count";
        delete g;
        return LV_ERR_PARSE;
      }
      g->off[(size_t)src[i] + 1]++;
      if (src[i] != dst[i]) g->off[(size_t)dst[i] + 1]++;
    }
    uint32_t max_deg = 0;
    for (uint32_t v = 0; v < n; v++) {
      const uint64_t d = g->off[(size_t)v + 1];
      if (d > max_deg) max_deg = (uint32_t)std::min<uint64_t>(d, 0xFFFFFFFFu);
      g->off[(size_t)v + 1] += g->off[v];
    }
    g->max_deg = max_deg;
    g->nnz = g->off[n];
    g->col.resize(g->nnz);
    g->w.resize(g->nnz);
    std::vector<uint64_t> cur(g->off.begin(), g->off.end() - 1);
    for (uint64_t i = 0; i < m; i++) {
      const uint32_t a = src[i], b = dst[i];
      const float x = w ? w[i] : 1.0f;
      uint64_t p = cur[a]++;
      g->col[p] = b;
      g->w[p] = x;
      if (a != b) {
        p = cur[b]++;
        g->col[p] = a;
        g->w[p] = x;
      }
    }
  } catch (const std::bad_alloc&) {
    delete g;
    return LV_ERR_NOMEM;
  }
  *out = g;
  return LV_OK;
}

// Parses a Matrix Market file into its edge lines (0-based indices, |w|,
// a weightless line repeating the previous weight), validated against the
// size line's vertex count.
lv_status lvb_parse_mtx(const char* path, uint32_t* n_out, std::vector<uint32_t>& src,
                        std::vector<uint32_t>& dst, std::vector<float>& ws) {
  FILE* f = fopen(path, "rb");
  if (!f) return io_fail(LV_ERR_IO, "Error opening file");
  std::string data;
  {
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    if (sz < 0) {
      fclose(f);
      return io_fail(LV_ERR_IO, "Error opening file");
    }
    try {
      data.resize((size_t)sz);
    } catch (const std::bad_alloc&) {
      fclose(f);
      return io_fail(LV_ERR_NOMEM, "file too large for host memory");
    }
    size_t got = fread(&data[0], 1, (size_t)sz, f);
    fclose(f);
    data.resize(got);
  }
  const char* p = data.data();
  const char* end = p + data.size();
  auto next_line = [&](const char*& ls, const char*& le) -> bool {
    if (p >= end) return false;
    ls = p;
    const char* nl = (const char*)memchr(p, '\n', (size_t)(end - p));
    le = nl ? nl : end;
    p = nl ? nl + 1 : end;
    return true;
  };
  const char *ls = nullptr, *le = nullptr;
  long lineno = 0;
  for (;;) {
    if (!next_line(ls, le)) return io_fail(LV_ERR_PARSE, "missing size line");
    lineno++;
    if (ls == le || *ls != '%') break;
  }
  uint64_t rows = 0, cols = 0, nnz = 0;
  {
    const char* q = ls;
    if (!parse_u64(q, le, &rows) || !parse_u64(q, le, &cols) || !parse_u64(q, le, &nnz))
      return io_fail(LV_ERR_PARSE, "bad size line (line " + std::to_string(lineno) + ")");
  }
  (void)rows;
  if (cols >= 0xFFFFFFFFull) return io_fail(LV_ERR_LIMIT, "vertex count must be < 2^32-1");
  try {
    src.resize(nnz);
    dst.resize(nnz);
    ws.resize(nnz);
  } catch (const std::bad_alloc&) {
    return io_fail(LV_ERR_NOMEM, "entry count too large for host memory");
  }
  // Entry lines are parsed in parallel: the body is cut at line ends into
  // chunks, a first sweep counts each chunk's lines (global line numbers),
  // a second parses the first nnz lines in place.  A line without a weight
  // repeats the previous line's (the reference's stream leaves `weight` as
  // it was), so each chunk's leading weightless lines are fixed up after.
  const char* body = p;
  const size_t body_len = (size_t)(end - body);
  unsigned hw = std::thread::hardware_concurrency();
  const unsigned nt = (unsigned)std::max<size_t>(
      1, std::min<size_t>({(size_t)std::min(hw ? hw : 1u, 32u), body_len / (1u << 22) + 1}));
  std::vector<const char*> cb(nt + 1);
  cb[0] = body;
  cb[nt] = end;
  for (unsigned t = 1; t < nt; t++) {
    const char* c = body + body_len * t / nt;
    if (c < cb[t - 1]) c = cb[t - 1];
    const char* nl = (const char*)memchr(c, '\n', (size_t)(end - c));
    cb[t] = nl ? nl + 1 : end;
  }
  std::vector<uint64_t> lines(nt + 1, 0);
  auto count_lines = [&](unsigned t) {
    uint64_t c = 0;
    const char* q = cb[t];
    while (q < cb[t + 1]) {
      const char* nl = (const char*)memchr(q, '\n', (size_t)(cb[t + 1] - q));
      c++;
      q = nl ? nl + 1 : cb[t + 1];
    }
    lines[t + 1] = c;
  };
  struct ChunkOut {
    bool zero = false;
    bool any_weight = false;
    uint64_t lead = 0;   // leading lines without a weight
    float last = 1.0f;   // last explicit weight of the chunk
    uint64_t bad = UINT64_MAX;  // first malformed line (global index)
    lv_status bad_status = LV_OK;
    std::string bad_what;
  };
  std::vector<ChunkOut> co(nt);
  auto parse_chunk = [&](unsigned t) {
    ChunkOut& o = co[t];
    uint64_t idx = lines[t];
    const char* q0 = cb[t];
    float wprev = 1.0f;
    while (q0 < cb[t + 1] && idx < nnz) {
      const char* nl = (const char*)memchr(q0, '\n', (size_t)(cb[t + 1] - q0));
      const char* le2 = nl ? nl : cb[t + 1];
      const char* q = q0;
      uint64_t a, b;
      if (!parse_u64(q, le2, &a) || !parse_u64(q, le2, &b)) {
        o.bad = idx;
        o.bad_status = LV_ERR_PARSE;
        o.bad_what = "bad entry line";
        return;
      }
      if (a > 0xFFFFFFFFull || b > 0xFFFFFFFFull) {
        o.bad = idx;
        o.bad_status = LV_ERR_PARSE;
        o.bad_what = "vertex index out of range";
        return;
      }
      float x;
      const int r = parse_weight(q, le2, &x);
      if (r < 0) {
        o.bad = idx;
        o.bad_status = LV_ERR_PARSE;
        o.bad_what = "bad weight";
        return;
      }
      if (r > 0) {
        wprev = std::fabs(x);
        o.any_weight = true;
        o.last = wprev;
      } else if (!o.any_weight) {
        o.lead++;
      }
      if (a == 0 || b == 0) o.zero = true;
      src[idx] = (uint32_t)a;
      dst[idx] = (uint32_t)b;
      ws[idx] = wprev;
      idx++;
      q0 = nl ? nl + 1 : cb[t + 1];
    }
  };
  auto run = [&](auto&& fn) {
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; t++) th.emplace_back(fn, t);
    fn(0u);
    for (auto& x : th) x.join();
  };
  try {
    run(count_lines);
    for (unsigned t = 0; t < nt; t++) lines[t + 1] += lines[t];
    if (lines[nt] < nnz)
      return io_fail(LV_ERR_PARSE, "fewer entry lines than the size line's count");
    run(parse_chunk);
  } catch (const std::system_error&) {
    return io_fail(LV_ERR_NOMEM, "parser threads could not start");
  }
  bool zero_based = false;
  float carry = 1.0f;
  for (unsigned t = 0; t < nt; t++) {
    const ChunkOut& o = co[t];
    if (o.bad != UINT64_MAX)  // the first failure in file order
      return io_fail(o.bad_status, o.bad_what + " (line " +
                                       std::to_string(lineno + o.bad + 1) + ")");
    zero_based = zero_based || o.zero;
    const uint64_t first = lines[t];
    const uint64_t stop = std::min<uint64_t>(first + o.lead, nnz);
    for (uint64_t k = first; k < stop; k++) ws[k] = carry;
    if (o.any_weight) carry = o.last;
  }
  const uint32_t n = (uint32_t)cols;
  for (uint64_t i = 0; i < nnz; i++) {
    if (!zero_based) {
      src[i]--;
      dst[i]--;
    }
    if (src[i] >= n || dst[i] >= n)
      return io_fail(LV_ERR_PARSE, "vertex index exceeds the size line's count");
  }
  *n_out = n;
  return LV_OK;
}

extern "C" {

lv_status lv_graph_load_mtx(const char* path, lv_graph** out) {
  if (!path || !out) return io_fail(LV_ERR_ARG, "NULL argument");
  *out = nullptr;
  uint32_t n = 0;
  std::vector<uint32_t> src, dst;
  std::vector<float> ws;
  lv_status s = lvb_parse_mtx(path, &n, src, dst, ws);
  if (s != LV_OK) return s;
  std::string err;
  s = lvb_graph_build(n, src.size(), src.data(), dst.data(), ws.data(), out, &err);
  if (s != LV_OK) return io_fail(s, err.empty() ? "graph construction failed" : err);
  return LV_OK;
}

lv_status lv_graph_from_edges(uint32_t n, uint64_t m, const uint32_t* src,
                              const uint32_t* dst, const float* weights,
                              lv_graph** out) {
  if (!out || (m && (!src || !dst))) return io_fail(LV_ERR_ARG, "NULL argument");
  if (n >= 0xFFFFFFFFu) return io_fail(LV_ERR_LIMIT, "vertex count must be < 2^32-1");
  *out = nullptr;
  std::vector<float> wabs;
  if (weights) {
    try {
      wabs.resize(m);
    } catch (const std::bad_alloc&) {
      return io_fail(LV_ERR_NOMEM, "out of host memory");
    }
    for (uint64_t i = 0; i < m; i++) wabs[i] = std::fabs(weights[i]);
  }
  std::string err;
  lv_status s = lvb_graph_build(n, m, src, dst, weights ? wabs.data() : nullptr, out, &err);
  if (s != LV_OK) return io_fail(s, err.empty() ? "graph construction failed" : err);
  return LV_OK;
}

lv_status lv_graph_from_csr(uint32_t n, const uint64_t* off, const uint32_t* col,
                            const float* w, lv_graph** out) {
  if (!out || !off) return io_fail(LV_ERR_ARG, "NULL argument");
  if (n >= 0xFFFFFFFFu) return io_fail(LV_ERR_LIMIT, "vertex count must be < 2^32-1");
  *out = nullptr;
  if (off[0] != 0) return io_fail(LV_ERR_ARG, "offsets must start at 0");
  for (uint32_t v = 0; v < n; v++)
    if (off[v + 1] < off[v]) return io_fail(LV_ERR_ARG, "offsets must be non-decreasing");
  const uint64_t nnz = off[n];
  if (nnz && (!col || !w)) return io_fail(LV_ERR_ARG, "NULL cols or weights");
  for (uint64_t j = 0; j < nnz; j++)
    if (col[j] >= n) return io_fail(LV_ERR_ARG, "column index out of range");
  lv_graph* g = new (std::nothrow) lv_graph();
  if (!g) return io_fail(LV_ERR_NOMEM, "out of host memory");
  try {
    g->n = n;
    g->nnz = nnz;
    g->off.assign(off, off + (size_t)n + 1);
    g->col.assign(col, col + nnz);
    g->w.assign(w, w + nnz);
    uint64_t md = 0;
    for (uint32_t v = 0; v < n; v++) md = std::max<uint64_t>(md, off[v + 1] - off[v]);
    g->max_deg = (uint32_t)std::min<uint64_t>(md, 0xFFFFFFFFu);
  } catch (const std::bad_alloc&) {
    delete g;
    return io_fail(LV_ERR_NOMEM, "out of host memory");
  }
  *out = g;
  return LV_OK;
}

lv_status lv_graph_view(const lv_graph* g, uint32_t* n, uint64_t* nnz,
                        const uint64_t** off, const uint32_t** col, const float** w,
                        uint32_t* max_deg) {
  if (!g) return io_fail(LV_ERR_ARG, "NULL graph");
  if (n) *n = g->n;
  if (nnz) *nnz = g->nnz;
  if (off) *off = g->off.data();
  if (col) *col = g->col.data();
  if (w) *w = g->w.data();
  if (max_deg) *max_deg = g->max_deg;
  return LV_OK;
}

// Binary CSR file: "LVBCSR01", n (u32), max degree (u32), nnz (u64), then
// offsets (u64, n+1), cols (u32, nnz), weights (f32, nnz); little-endian.
static const char kCsrMagic[8] = {'L', 'V', 'B', 'C', 'S', 'R', '0', '1'};

lv_status lv_graph_save(const lv_graph* g, const char* path) {
  if (!g || !path) return io_fail(LV_ERR_ARG, "NULL argument");
  FILE* f = fopen(path, "wb");
  if (!f) return io_fail(LV_ERR_IO, "cannot open file for writing");
  const uint32_t hdr32[2] = {g->n, g->max_deg};
  const uint64_t nnz = g->nnz;
  bool ok = fwrite(kCsrMagic, 1, 8, f) == 8 && fwrite(hdr32, 4, 2, f) == 2 &&
            fwrite(&nnz, 8, 1, f) == 1 &&
            fwrite(g->off.data(), 8, (size_t)g->n + 1, f) == (size_t)g->n + 1 &&
            fwrite(g->col.data(), 4, nnz, f) == nnz && fwrite(g->w.data(), 4, nnz, f) == nnz;
  ok = (fclose(f) == 0) && ok;
  if (!ok) return io_fail(LV_ERR_IO, "write failed");
  return LV_OK;
}

lv_status lv_graph_load(const char* path, lv_graph** out) {
  if (!path || !out) return io_fail(LV_ERR_ARG, "NULL argument");
  *out = nullptr;
  FILE* f = fopen(path, "rb");
  if (!f) return io_fail(LV_ERR_IO, "Error opening file");
  char magic[8];
  uint32_t hdr32[2];
  uint64_t nnz = 0;
  if (fread(magic, 1, 8, f) != 8 || memcmp(magic, kCsrMagic, 8) != 0 ||
      fread(hdr32, 4, 2, f) != 2 || fread(&nnz, 8, 1, f) != 1 || hdr32[0] == 0xFFFFFFFFu) {
    fclose(f);
    return io_fail(LV_ERR_PARSE, "not a binary CSR file");
  }
  lv_graph* g = new (std::nothrow) lv_graph();
  if (!g) {
    fclose(f);
    return io_fail(LV_ERR_NOMEM, "graph allocation failed");
  }
  const uint32_t n = hdr32[0];
  try {
    g->n = n;
    g->max_deg = hdr32[1];
    g->nnz = nnz;
    g->off.resize((size_t)n + 1);
    g->col.resize(nnz);
    g->w.resize(nnz);
  } catch (const std::bad_alloc&) {
    fclose(f);
    delete g;
    return io_fail(LV_ERR_NOMEM, "graph too large for host memory");
  }
  bool ok = fread(g->off.data(), 8, (size_t)n + 1, f) == (size_t)n + 1 &&
            fread(g->col.data(), 4, nnz, f) == nnz && fread(g->w.data(), 4, nnz, f) == nnz;
  fclose(f);
  // the structure must be a valid CSR of n vertices
  ok = ok && g->off[0] == 0 && g->off[n] == nnz;
  for (uint32_t v = 0; ok && v < n; v++) ok = g->off[v] <= g->off[(size_t)v + 1];
  for (uint64_t j = 0; ok && j < nnz; j++) ok = g->col[j] < n;
  if (!ok) {
    delete g;
    return io_fail(LV_ERR_PARSE, "truncated or inconsistent binary CSR file");
  }
  *out = g;
  return LV_OK;
}

void lv_graph_destroy(lv_graph* g) { delete g; }

}  // extern "C"
