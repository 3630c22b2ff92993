// Host side of the graph boundary: the text format, per-graph CSR
// construction and batching with global ids.  Behaviour follows the
// reference's IntermediateGraph / toCSRGraph / createDeviceCSRGraph
// (library/include/graph.hpp:151-314) and io::loadCSRGraphsFromFile
// (library/include/io.hpp:46-55); the code is this library's own.
#include <algorithm>
#include <cerrno>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.hpp"
#include "host_graphs.hpp"

namespace sigmo_b200 {

namespace {
thread_local std::string g_last_error;
}

void set_error_message(const char* msg) { g_last_error = msg ? msg : ""; }
const char* get_error_message() { return g_last_error.c_str(); }

bool alloc_host_graphs(sigmo_host_graphs* g, uint32_t num_graphs, uint64_t total_nodes, uint64_t total_edges) {
  std::memset(g, 0, sizeof(*g));
  g->num_graphs = num_graphs;
  g->total_nodes = total_nodes;
  g->total_edges = total_edges;
  g->graph_offsets = static_cast<uint32_t*>(std::malloc(sizeof(uint32_t) * (num_graphs + 1ull)));
  g->row_offsets = static_cast<uint32_t*>(std::malloc(sizeof(uint32_t) * (total_nodes + 1ull)));
  g->column_indices = static_cast<uint32_t*>(std::malloc(sizeof(uint32_t) * std::max<uint64_t>(total_edges, 1)));
  g->node_labels = static_cast<uint8_t*>(std::malloc(std::max<uint64_t>(total_nodes, 1)));
  g->edge_labels = static_cast<uint8_t*>(std::malloc(std::max<uint64_t>(total_edges, 1)));
  if (!g->graph_offsets || !g->row_offsets || !g->column_indices || !g->node_labels || !g->edge_labels) {
    sigmo_host_graphs_free(g);
    return false;
  }
  return true;
}

// ---- per-graph CSR (toCSRGraph, graph.hpp:216-247) ------------------------
// Undirected edges become two directed entries; a vertex's neighbours appear
// in input-edge order.  A self-loop (a, a) advances the vertex's cursor twice
// but writes one slot, leaving the second slot as (0, 0): the reference's
// behaviour, kept so that every input maps to the same CSR.
void to_csr(const TextGraph& tg, LocalCSR* out) {
  const uint32_t n = tg.num_nodes;
  out->num_nodes = n;
  out->node_labels = tg.node_labels;
  out->row_offsets.assign(n + 1ull, 0u);
  for (const auto& e : tg.edges) {
    out->row_offsets[e.u + 1]++;
    out->row_offsets[e.v + 1]++;
  }
  for (size_t i = 1; i < out->row_offsets.size(); ++i) out->row_offsets[i] += out->row_offsets[i - 1];
  const uint32_t nnz = out->row_offsets.back();
  out->column_indices.assign(nnz, 0u);
  out->edge_labels.assign(nnz, 0u);
  std::vector<uint32_t> cur(n + 1ull, 0u);
  for (const auto& e : tg.edges) {
    out->column_indices[out->row_offsets[e.u] + cur[e.u]] = e.v;
    out->edge_labels[out->row_offsets[e.u] + cur[e.u]] = e.label;
    out->column_indices[out->row_offsets[e.v] + cur[e.v]] = e.u;
    out->edge_labels[out->row_offsets[e.v] + cur[e.v]] = e.label;
    cur[e.u]++;
    cur[e.v]++;
  }
}

// ---- batching (createDeviceCSRGraph host part, graph.hpp:255-294) ---------
int batch_graphs(const std::vector<LocalCSR>& graphs, sigmo_host_graphs* out) {
  uint64_t total_nodes = 0, total_edges = 0;
  for (const auto& g : graphs) {
    total_nodes += g.num_nodes;
    total_edges += g.row_offsets.empty() ? 0 : g.row_offsets.back();
  }
  if (total_nodes >= 0xFFFFFFFFull || total_edges >= 0xFFFFFFFFull || graphs.size() >= 0xFFFFFFFFull)
    return fail(SIGMO_ERR_DOMAIN, "batch exceeds 32-bit vertex/edge ids (%llu vertices, %llu entries)",
                (unsigned long long)total_nodes, (unsigned long long)total_edges);
  if (!alloc_host_graphs(out, static_cast<uint32_t>(graphs.size()), total_nodes, total_edges))
    return fail(SIGMO_ERR_OOM, "host allocation of a %llu-vertex batch failed", (unsigned long long)total_nodes);
  uint64_t vo = 0, eo = 0;
  out->graph_offsets[0] = 0;
  out->row_offsets[0] = 0;
  for (size_t gi = 0; gi < graphs.size(); ++gi) {
    const auto& g = graphs[gi];
    const uint32_t n = g.num_nodes;
    const uint32_t nnz = g.row_offsets.empty() ? 0 : g.row_offsets.back();
    out->graph_offsets[gi + 1] = static_cast<uint32_t>(vo + n);
    for (uint32_t j = 0; j <= n; ++j) out->row_offsets[vo + j] = static_cast<uint32_t>(g.row_offsets[j] + eo);
    for (uint32_t j = 0; j < nnz; ++j) {
      out->column_indices[eo + j] = static_cast<uint32_t>(g.column_indices[j] + vo);
      out->edge_labels[eo + j] = g.edge_labels[j];
    }
    if (n) std::memcpy(out->node_labels + vo, g.node_labels.data(), n);
    vo += n;
    eo += nnz;
  }
  return SIGMO_OK;
}

// ---- text format (IntermediateGraph(line), graph.hpp:154-206) -------------
namespace {

struct Tokenizer {
  const char* p;
  const char* end;
  bool next(const char** tok, size_t* len) {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n' || *p == '\v' || *p == '\f')) ++p;
    if (p >= end) return false;
    const char* s = p;
    while (p < end && !(*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n' || *p == '\v' || *p == '\f')) ++p;
    *tok = s;
    *len = static_cast<size_t>(p - s);
    return true;
  }
};

bool parse_ulong(const char* s, size_t len, unsigned long long* v) {
  if (len == 0 || len > 24) return false;
  char buf[32];
  std::memcpy(buf, s, len);
  buf[len] = 0;
  char* endp = nullptr;
  errno = 0;
  unsigned long long x = std::strtoull(buf, &endp, 10);
  if (errno || endp == buf) return false;
  *v = x;
  return true;
}
bool parse_long(const char* s, size_t len, long long* v) {
  if (len == 0 || len > 24) return false;
  char buf[32];
  std::memcpy(buf, s, len);
  buf[len] = 0;
  char* endp = nullptr;
  errno = 0;
  long long x = std::strtoll(buf, &endp, 10);
  if (errno || endp == buf) return false;
  *v = x;
  return true;
}

}  // namespace

int parse_line(const char* line, size_t len, TextGraph* out) {
  Tokenizer tk{line, line + len};
  const char* t;
  size_t tl;
  unsigned long long n, nl, ne;
  if (!tk.next(&t, &tl) || tl < 3 || !parse_ulong(t + 2, tl - 2, &n)) return fail(SIGMO_ERR_FORMAT, "Invalid graph format: bad n# token");
  if (!tk.next(&t, &tl) || tl < 3 || !parse_ulong(t + 2, tl - 2, &nl)) return fail(SIGMO_ERR_FORMAT, "Invalid graph format: bad l# token");
  if (n >= 0xFFFFFFFFull) return fail(SIGMO_ERR_DOMAIN, "graph with %llu vertices", n);
  out->num_nodes = static_cast<uint32_t>(n);
  out->max_labels = static_cast<uint32_t>(nl);
  out->node_labels.assign(n, 0u);
  out->edges.clear();
  for (unsigned long long i = 0; i < n; ++i) {
    unsigned long long node;
    long long lab;
    if (!tk.next(&t, &tl) || !parse_ulong(t, tl, &node)) return fail(SIGMO_ERR_FORMAT, "Invalid graph format: vertex id");
    if (!tk.next(&t, &tl) || !parse_long(t, tl, &lab)) return fail(SIGMO_ERR_FORMAT, "Invalid graph format: vertex label");
    if (node >= n) return fail(SIGMO_ERR_FORMAT, "Invalid graph format: vertex id %llu >= n#%llu", node, n);
    out->node_labels[node] = static_cast<uint8_t>(lab);  // int -> uint8_t, as label_t
  }
  if (!tk.next(&t, &tl) || tl < 3 || !parse_ulong(t + 2, tl - 2, &ne)) return fail(SIGMO_ERR_FORMAT, "Invalid graph format: bad e# token");
  std::vector<std::pair<const char*, size_t>> toks;
  while (tk.next(&t, &tl)) toks.emplace_back(t, tl);
  size_t stride;
  if (toks.size() == ne * 3) stride = 3;
  else if (toks.size() == ne * 2) stride = 2;
  else return fail(SIGMO_ERR_FORMAT, "Invalid graph format");
  out->edges.resize(ne);
  for (unsigned long long i = 0; i < ne; ++i) {
    unsigned long long u, v;
    long long lab = 0;
    if (!parse_ulong(toks[i * stride].first, toks[i * stride].second, &u) ||
        !parse_ulong(toks[i * stride + 1].first, toks[i * stride + 1].second, &v))
      return fail(SIGMO_ERR_FORMAT, "Invalid graph format: edge endpoint");
    if (stride == 3 && !parse_long(toks[i * stride + 2].first, toks[i * stride + 2].second, &lab))
      return fail(SIGMO_ERR_FORMAT, "Invalid graph format: edge label");
    if (u >= n || v >= n) return fail(SIGMO_ERR_FORMAT, "Invalid graph format: edge (%llu, %llu) outside n#%llu", u, v, n);
    out->edges[i] = {static_cast<uint32_t>(u), static_cast<uint32_t>(v), static_cast<uint8_t>(lab)};
  }
  return SIGMO_OK;
}

void format_graph(const TextGraph& g, std::string* s) {
  char buf[64];
  std::snprintf(buf, sizeof(buf), "n#%u l#%u ", g.num_nodes, g.max_labels);
  *s += buf;
  for (uint32_t i = 0; i < g.num_nodes; ++i) {
    std::snprintf(buf, sizeof(buf), "%u %u ", i, static_cast<unsigned>(g.node_labels[i]));
    *s += buf;
  }
  std::snprintf(buf, sizeof(buf), "e#%zu ", g.edges.size());
  *s += buf;
  for (const auto& e : g.edges) {
    std::snprintf(buf, sizeof(buf), "%u %u %u ", e.u, e.v, static_cast<unsigned>(e.label));
    *s += buf;
  }
  *s += "\n";
}

}  // namespace sigmo_b200

using namespace sigmo_b200;

extern "C" {

const char* sigmo_last_error(void) { return get_error_message(); }
const char* sigmo_version(void) { return "sigmo_b200 0.1.0 (sm_100a)"; }

void sigmo_host_graphs_free(sigmo_host_graphs* g) {
  if (!g) return;
  std::free(g->graph_offsets);
  std::free(g->row_offsets);
  std::free(g->column_indices);
  std::free(g->node_labels);
  std::free(g->edge_labels);
  std::memset(g, 0, sizeof(*g));
}

int sigmo_parse_graphs(const char* text, size_t len, sigmo_host_graphs* out) {
  if (!out || (!text && len)) return fail(SIGMO_ERR_INVALID, "sigmo_parse_graphs: null argument");
  std::memset(out, 0, sizeof(*out));
  std::vector<LocalCSR> graphs;
  size_t pos = 0;
  TextGraph tg;
  while (pos < len) {
    size_t e = pos;
    while (e < len && text[e] != '\n') ++e;
    bool blank = true;
    for (size_t i = pos; i < e; ++i)
      if (!(text[i] == ' ' || text[i] == '\t' || text[i] == '\r')) {
        blank = false;
        break;
      }
    if (!blank) {
      int rc = parse_line(text + pos, e - pos, &tg);
      if (rc) return rc;
      graphs.emplace_back();
      to_csr(tg, &graphs.back());
    }
    pos = e + 1;
  }
  return batch_graphs(graphs, out);
}

int sigmo_host_graphs_concat(const sigmo_host_graphs* a, const sigmo_host_graphs* b, sigmo_host_graphs* out) {
  if (!a || !b || !out) return fail(SIGMO_ERR_INVALID, "sigmo_host_graphs_concat: null argument");
  uint64_t n = a->total_nodes + b->total_nodes, m = a->total_edges + b->total_edges;
  uint64_t G = static_cast<uint64_t>(a->num_graphs) + b->num_graphs;
  if (n >= 0xFFFFFFFFull || m >= 0xFFFFFFFFull || G >= 0xFFFFFFFFull) return fail(SIGMO_ERR_DOMAIN, "concatenation exceeds 32-bit ids");
  if (!alloc_host_graphs(out, static_cast<uint32_t>(G), n, m)) return fail(SIGMO_ERR_OOM, "host allocation failed");
  std::memcpy(out->graph_offsets, a->graph_offsets, sizeof(uint32_t) * (a->num_graphs + 1ull));
  for (uint32_t i = 1; i <= b->num_graphs; ++i)
    out->graph_offsets[a->num_graphs + i] = static_cast<uint32_t>(b->graph_offsets[i] + a->total_nodes);
  std::memcpy(out->row_offsets, a->row_offsets, sizeof(uint32_t) * a->total_nodes);
  for (uint64_t i = 0; i <= b->total_nodes; ++i)
    out->row_offsets[a->total_nodes + i] = static_cast<uint32_t>(b->row_offsets[i] + a->total_edges);
  if (a->total_edges) {
    std::memcpy(out->column_indices, a->column_indices, sizeof(uint32_t) * a->total_edges);
    std::memcpy(out->edge_labels, a->edge_labels, a->total_edges);
  }
  for (uint64_t i = 0; i < b->total_edges; ++i) {
    out->column_indices[a->total_edges + i] = static_cast<uint32_t>(b->column_indices[i] + a->total_nodes);
    out->edge_labels[a->total_edges + i] = b->edge_labels[i];
  }
  if (a->total_nodes) std::memcpy(out->node_labels, a->node_labels, a->total_nodes);
  if (b->total_nodes) std::memcpy(out->node_labels + a->total_nodes, b->node_labels, b->total_nodes);
  return SIGMO_OK;
}

int sigmo_host_graphs_slice(const sigmo_host_graphs* in, uint32_t first, uint32_t count, sigmo_host_graphs* out) {
  if (!in || !out) return fail(SIGMO_ERR_INVALID, "sigmo_host_graphs_slice: null argument");
  if (static_cast<uint64_t>(first) + count > in->num_graphs) return fail(SIGMO_ERR_INVALID, "slice [%u, %u) outside %u graphs", first, first + count, in->num_graphs);
  const uint32_t v0 = in->graph_offsets[first], v1 = in->graph_offsets[first + count];
  const uint32_t e0 = in->row_offsets[v0], e1 = in->row_offsets[v1];
  if (!alloc_host_graphs(out, count, v1 - v0, e1 - e0)) return fail(SIGMO_ERR_OOM, "host allocation failed");
  for (uint32_t i = 0; i <= count; ++i) out->graph_offsets[i] = in->graph_offsets[first + i] - v0;
  for (uint32_t i = 0; i <= v1 - v0; ++i) out->row_offsets[i] = in->row_offsets[v0 + i] - e0;
  for (uint32_t i = 0; i < e1 - e0; ++i) {
    out->column_indices[i] = in->column_indices[e0 + i] - v0;
    out->edge_labels[i] = in->edge_labels[e0 + i];
  }
  if (v1 > v0) std::memcpy(out->node_labels, in->node_labels + v0, v1 - v0);
  return SIGMO_OK;
}

int sigmo_format_graphs(const sigmo_host_graphs* in, char* buf, size_t* len) {
  if (!in || !len) return fail(SIGMO_ERR_INVALID, "sigmo_format_graphs: null argument");
  // Each undirected edge is emitted once, from the CSR entry (u -> v) with
  // u <= v, in CSR order; parsing the text back gives the same topology and
  // labels (neighbour order within a row may differ from the original input).
  std::string s;
  for (uint32_t g = 0; g < in->num_graphs; ++g) {
    TextGraph tg;
    const uint32_t v0 = in->graph_offsets[g], v1 = in->graph_offsets[g + 1];
    tg.num_nodes = v1 - v0;
    tg.max_labels = 11;
    tg.node_labels.assign(in->node_labels + v0, in->node_labels + v1);
    for (uint32_t u = v0; u < v1; ++u)
      for (uint32_t i = in->row_offsets[u]; i < in->row_offsets[u + 1]; ++i) {
        uint32_t v = in->column_indices[i];
        if (u <= v) tg.edges.push_back({u - v0, v - v0, in->edge_labels[i]});
      }
    format_graph(tg, &s);
  }
  if (buf) {
    if (*len < s.size()) return fail(SIGMO_ERR_INVALID, "sigmo_format_graphs: buffer of %zu bytes < %zu", *len, s.size());
    std::memcpy(buf, s.data(), s.size());
  }
  *len = s.size();
  return SIGMO_OK;
}

// ---- binary batches ---------------------------------------------------------
// Layout (little-endian): "SIGMOCSR", u32 version (1), u32 num_graphs,
// u64 total_nodes, u64 total_edges, then graph_offsets[G+1], row_offsets[N+1],
// column_indices[E] (u32), node_labels[N], edge_labels[E] (u8).  Loading
// checks every size and offset, so a damaged file is an error, not a batch.
int sigmo_graphs_save(const sigmo_host_graphs* in, const char* path) {
  if (!in || !path) return fail(SIGMO_ERR_INVALID, "sigmo_graphs_save: null argument");
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(SIGMO_ERR_INVALID, "cannot open %s for writing", path);
  const char magic[8] = {'S', 'I', 'G', 'M', 'O', 'C', 'S', 'R'};
  const uint32_t head[2] = {1u, in->num_graphs};
  const uint64_t sizes[2] = {in->total_nodes, in->total_edges};
  bool ok = std::fwrite(magic, 1, 8, f) == 8 && std::fwrite(head, 4, 2, f) == 2 && std::fwrite(sizes, 8, 2, f) == 2;
  auto put = [&](const void* p, size_t elem, uint64_t n) {
    if (ok && n) ok = std::fwrite(p, elem, n, f) == n;
  };
  put(in->graph_offsets, 4, in->num_graphs + 1ull);
  put(in->row_offsets, 4, in->total_nodes + 1);
  put(in->column_indices, 4, in->total_edges);
  put(in->node_labels, 1, in->total_nodes);
  put(in->edge_labels, 1, in->total_edges);
  ok = (std::fclose(f) == 0) && ok;
  return ok ? SIGMO_OK : fail(SIGMO_ERR_INVALID, "writing %s failed", path);
}

int sigmo_graphs_load(const char* path, sigmo_host_graphs* out) {
  if (!path || !out) return fail(SIGMO_ERR_INVALID, "sigmo_graphs_load: null argument");
  std::memset(out, 0, sizeof(*out));
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(SIGMO_ERR_INVALID, "cannot open %s", path);
  char magic[8];
  uint32_t head[2];
  uint64_t sizes[2];
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "SIGMOCSR", 8) == 0 && std::fread(head, 4, 2, f) == 2 &&
            head[0] == 1u && std::fread(sizes, 8, 2, f) == 2 && sizes[0] < (1ull << 32) && sizes[1] < (1ull << 32);
  if (!ok) {
    std::fclose(f);
    return fail(SIGMO_ERR_FORMAT, "%s is not a sigmo_b200 binary batch (version 1)", path);
  }
  if (!alloc_host_graphs(out, head[1], sizes[0], sizes[1])) {
    std::fclose(f);
    return fail(SIGMO_ERR_OOM, "host allocation of a %llu-vertex batch failed", (unsigned long long)sizes[0]);
  }
  auto get = [&](void* p, size_t elem, uint64_t n) {
    if (ok && n) ok = std::fread(p, elem, n, f) == n;
  };
  get(out->graph_offsets, 4, out->num_graphs + 1ull);
  get(out->row_offsets, 4, out->total_nodes + 1);
  get(out->column_indices, 4, out->total_edges);
  get(out->node_labels, 1, out->total_nodes);
  get(out->edge_labels, 1, out->total_edges);
  std::fclose(f);
  // structural checks: offsets start at 0, never decrease and end at the
  // totals; neighbours stay inside their graph
  if (ok) ok = out->graph_offsets[0] == 0 && out->graph_offsets[out->num_graphs] == out->total_nodes && out->row_offsets[0] == 0 &&
               out->row_offsets[out->total_nodes] == out->total_edges;
  for (uint32_t g = 0; ok && g < out->num_graphs; ++g) {
    const uint32_t v0 = out->graph_offsets[g], v1 = out->graph_offsets[g + 1];
    if (v1 < v0) ok = false;
    for (uint32_t v = v0; ok && v < v1; ++v) {
      if (out->row_offsets[v + 1] < out->row_offsets[v]) ok = false;
      for (uint32_t i = out->row_offsets[v]; ok && i < out->row_offsets[v + 1]; ++i)
        if (out->column_indices[i] < v0 || out->column_indices[i] >= v1) ok = false;
    }
  }
  if (!ok) {
    sigmo_host_graphs_free(out);
    return fail(SIGMO_ERR_FORMAT, "%s is truncated or inconsistent", path);
  }
  return SIGMO_OK;
}

}  // extern "C"
