// Host-side graph containers shared by the parser, the batcher and the
// synthetic generator.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/sigmo_b200.h"

namespace sigmo_b200 {

struct TextEdge {
  uint32_t u, v;
  uint8_t label;
};

// One graph as read from a text line (IntermediateGraph, graph.hpp:151-252).
struct TextGraph {
  uint32_t num_nodes = 0;
  uint32_t max_labels = 0;
  std::vector<uint8_t> node_labels;
  std::vector<TextEdge> edges;
};

// One graph in local-id CSR form (CSRGraph, graph.hpp:37-60).
struct LocalCSR {
  uint32_t num_nodes = 0;
  std::vector<uint32_t> row_offsets;
  std::vector<uint32_t> column_indices;
  std::vector<uint8_t> node_labels;
  std::vector<uint8_t> edge_labels;
};

int parse_line(const char* line, size_t len, TextGraph* out);
void to_csr(const TextGraph& tg, LocalCSR* out);
int batch_graphs(const std::vector<LocalCSR>& graphs, sigmo_host_graphs* out);
void format_graph(const TextGraph& g, std::string* s);

}  // namespace sigmo_b200
