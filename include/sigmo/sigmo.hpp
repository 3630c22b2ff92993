// sigmo/sigmo.hpp — C++ host API of sigmo_b200, mirroring the reference's
// header-only `namespace sigmo` (library/include/sigmo.hpp:8-17) so that a
// driver written against SIGMo (library/src/sigmo.cpp) compiles against this
// header with `sycl::queue` replaced by `sigmo::Queue`.  Every call goes
// through the C ABI in sigmo_b200.h; errors throw std::runtime_error with the
// library's message (the reference throws on bad input, graph.hpp:204, and
// surfaces device errors through queue.wait_and_throw()).
//
// Link with: -I<repo>/include -L<repo>/sigmo_b200 -lsigmo_b200
#pragma once

#include <chrono>
#include <cstdint>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../sigmo_b200.h"

namespace sigmo {

inline void check(int rc) {
  if (rc != SIGMO_OK) throw std::runtime_error(std::string("sigmo_b200: ") + sigmo_last_error());
}

// ---- types (library/include/types.hpp:14-28) ------------------------------
namespace types {
using row_offset_t = uint32_t;
using col_index_t = uint32_t;
using label_t = uint8_t;
using node_t = uint32_t;
using adjacency_t = uint64_t;
using candidates_t = uint32_t;
constexpr label_t WILDCARD_NODE = 255;
constexpr node_t NULL_NODE = 0xFFFFFFFFu;
}  // namespace types

enum class CandidatesDomain { Query, Data };  // device.hpp:14 (Query is the only supported domain)
enum class Profile { RefPtx = SIGMO_PROFILE_REF_PTX, Exact = SIGMO_PROFILE_EXACT };

// ---- queue: replaces sycl::queue and device::DeviceOptions ------------------
class Queue {
 public:
  explicit Queue(int device = 0, Profile profile = Profile::RefPtx, uint32_t join_work_group_size = 128,
                 uint32_t filter_work_group_size = 512) {
    sigmo_options o;
    sigmo_default_options(&o);
    o.profile = static_cast<int>(profile);
    o.join_work_group_size = join_work_group_size;
    o.filter_work_group_size = filter_work_group_size;
    check(sigmo_queue_create(device, &o, &h_));
  }
  ~Queue() { sigmo_queue_destroy(h_); }
  Queue(const Queue&) = delete;
  Queue& operator=(const Queue&) = delete;
  void wait() { check(sigmo_queue_wait(h_)); }
  void wait_and_throw() { wait(); }
  sigmo_queue_t handle() const { return h_; }
  size_t global_mem_size() const {
    uint64_t m = 0;
    check(sigmo_queue_device_info(h_, &m, nullptr, 0));
    return m;
  }
  std::string device_name() const {
    char buf[256];
    check(sigmo_queue_device_info(h_, nullptr, buf, sizeof(buf)));
    return buf;
  }

 private:
  sigmo_queue_t h_ = nullptr;
};

// ---- utils::BatchedEvent (utils.hpp:127-161) ---------------------------------
namespace utils {
class BatchedEvent {
 public:
  BatchedEvent() = default;
  explicit BatchedEvent(Queue& q) : q_(&q) { check(sigmo_queue_last_stage_ms(q.handle(), &ms_)); }
  void wait() {
    if (q_) q_->wait();
  }
  std::chrono::duration<double> getProfilingInfo() const { return std::chrono::duration<double>(ms_ / 1e3); }

 private:
  Queue* q_ = nullptr;
  double ms_ = 0.0;
};
}  // namespace utils

// ---- host graphs (CSRGraph, graph.hpp:37-60) -----------------------------------
class CSRGraph {
 public:
  CSRGraph(std::vector<types::row_offset_t> row_offsets, std::vector<types::col_index_t> column_indices,
           std::vector<types::label_t> node_labels, std::vector<types::label_t> edge_labels, size_t num_nodes)
      : row_offsets_(std::move(row_offsets)), column_indices_(std::move(column_indices)),
        node_labels_(std::move(node_labels)), edge_labels_(std::move(edge_labels)), num_nodes_(num_nodes) {}
  const types::row_offset_t* getRowOffsets() const { return row_offsets_.data(); }
  const types::col_index_t* getColumnIndices() const { return column_indices_.data(); }
  const types::label_t* getNodeLabels() const { return node_labels_.data(); }
  const types::label_t* getEdgeLabels() const { return edge_labels_.data(); }
  size_t getNumNodes() const { return num_nodes_; }

 private:
  std::vector<types::row_offset_t> row_offsets_;
  std::vector<types::col_index_t> column_indices_;
  std::vector<types::label_t> node_labels_;
  std::vector<types::label_t> edge_labels_;
  size_t num_nodes_;
};

namespace detail {
// Splits a batched host set (global ids) back into per-graph CSRGraph objects.
inline std::vector<CSRGraph> unbatch(const sigmo_host_graphs& h) {
  std::vector<CSRGraph> out;
  out.reserve(h.num_graphs);
  for (uint32_t g = 0; g < h.num_graphs; ++g) {
    const uint32_t v0 = h.graph_offsets[g], v1 = h.graph_offsets[g + 1];
    const uint32_t e0 = h.row_offsets[v0], e1 = h.row_offsets[v1];
    std::vector<uint32_t> ro(v1 - v0 + 1), col(e1 - e0);
    for (uint32_t i = 0; i <= v1 - v0; ++i) ro[i] = h.row_offsets[v0 + i] - e0;
    for (uint32_t i = 0; i < e1 - e0; ++i) col[i] = h.column_indices[e0 + i] - v0;
    out.emplace_back(std::move(ro), std::move(col), std::vector<uint8_t>(h.node_labels + v0, h.node_labels + v1),
                     std::vector<uint8_t>(h.edge_labels + e0, h.edge_labels + e1), v1 - v0);
  }
  return out;
}
}  // namespace detail

// ---- io (io.hpp:46-55) -------------------------------------------------------
namespace io {
inline std::vector<CSRGraph> loadCSRGraphsFromLines(const std::vector<std::string>& lines) {
  std::string text;
  for (const auto& l : lines) text += l + "\n";
  sigmo_host_graphs h;
  check(sigmo_parse_graphs(text.data(), text.size(), &h));
  auto out = detail::unbatch(h);
  sigmo_host_graphs_free(&h);
  return out;
}
inline std::vector<CSRGraph> loadCSRGraphsFromFile(const std::string& filename) {
  std::ifstream f(filename);
  if (!f) throw std::runtime_error("cannot open " + filename);
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string text = ss.str();
  sigmo_host_graphs h;
  check(sigmo_parse_graphs(text.data(), text.size(), &h));
  auto out = detail::unbatch(h);
  sigmo_host_graphs_free(&h);
  return out;
}
}  // namespace io

// ---- DeviceBatchedCSRGraph (graph.hpp:62-112) ----------------------------------
struct DeviceBatchedCSRGraph {
  sigmo_graph_t handle = nullptr;
  uint32_t num_graphs = 0;
  size_t total_nodes = 0;
  size_t total_edges = 0;
};

// createDeviceCSRGraph (graph.hpp:255-314).  The graphs' own arrays are
// copied back to back (no per-element rebasing on the host) and the batch is
// assembled on the device (sigmo_graph_create_from_local; the reference
// concatenates on the host, graph.hpp:254).
inline DeviceBatchedCSRGraph createDeviceCSRGraph(Queue& queue, std::vector<CSRGraph>& graphs) {
  size_t N = 0, E = 0;
  for (auto& g : graphs) {
    N += g.getNumNodes();
    E += g.getRowOffsets()[g.getNumNodes()];
  }
  const size_t G = graphs.size();
  std::vector<uint32_t> nc(G), ec(G), ro, col;
  std::vector<uint8_t> nl, el;
  ro.reserve(N + G);
  col.reserve(E);
  nl.reserve(N);
  el.reserve(E);
  for (size_t gi = 0; gi < G; ++gi) {
    auto& g = graphs[gi];
    const size_t n = g.getNumNodes(), m = g.getRowOffsets()[n];
    nc[gi] = static_cast<uint32_t>(n);
    ec[gi] = static_cast<uint32_t>(m);
    ro.insert(ro.end(), g.getRowOffsets(), g.getRowOffsets() + n + 1);
    col.insert(col.end(), g.getColumnIndices(), g.getColumnIndices() + m);
    nl.insert(nl.end(), g.getNodeLabels(), g.getNodeLabels() + n);
    el.insert(el.end(), g.getEdgeLabels(), g.getEdgeLabels() + m);
  }
  DeviceBatchedCSRGraph d;
  check(sigmo_graph_create_from_local(queue.handle(), static_cast<uint32_t>(G), nc.data(), ec.data(), ro.data(), col.data(),
                                      nl.data(), el.data(), &d.handle));
  d.num_graphs = static_cast<uint32_t>(G);
  d.total_nodes = N;
  d.total_edges = E;
  return d;
}

inline void destroyDeviceCSRGraph(DeviceBatchedCSRGraph& g, Queue&) {
  sigmo_graph_destroy(g.handle);
  g.handle = nullptr;
}

inline size_t getDeviceGraphAllocSize(const DeviceBatchedCSRGraph& g) {
  uint64_t b = 0;
  check(sigmo_graph_alloc_size(g.handle, &b));
  return b;
}

// ---- candidates::Candidates (candidates.hpp:14-204) ------------------------------
namespace candidates {
class Candidates {
 public:
  // Host view returned by getHostCandidates (candidates.hpp:185-190).
  struct CandidatesHost {
    std::vector<types::candidates_t> candidates;
    size_t source_nodes = 0, target_nodes = 0, single_node_size = 0;
    bool contains(types::node_t s, types::node_t c) const {
      return (candidates[s * single_node_size + c / 32] >> (c % 32)) & 1u;
    }
    uint32_t getCandidatesCount(types::node_t s) const {
      uint32_t n = 0;
      for (size_t i = 0; i < single_node_size; ++i) n += __builtin_popcount(candidates[s * single_node_size + i]);
      return n;
    }
  };
  Candidates(Queue& queue, size_t source_nodes, size_t target_nodes) : source_(source_nodes), target_(target_nodes) {
    check(sigmo_candidates_create(queue.handle(), source_nodes, target_nodes, &h_));
  }
  ~Candidates() { sigmo_candidates_destroy(h_); }
  Candidates(const Candidates&) = delete;
  Candidates& operator=(const Candidates&) = delete;
  CandidatesHost getHostCandidates() const {
    CandidatesHost c;
    c.source_nodes = source_;
    c.target_nodes = target_;
    c.single_node_size = (target_ + 31) / 32;
    c.candidates.resize(source_ * c.single_node_size);
    check(sigmo_candidates_download(h_, 0, source_, c.candidates.data()));
    return c;
  }
  std::vector<uint32_t> getCandidatesCounts() const {
    std::vector<uint32_t> v(source_);
    check(sigmo_candidates_row_counts(h_, v.data()));
    return v;
  }
  size_t getAllocationSize() const {
    uint64_t b = 0;
    check(sigmo_candidates_alloc_size(h_, &b));
    return b;
  }
  sigmo_candidates_t handle() const { return h_; }

 private:
  sigmo_candidates_t h_ = nullptr;
  size_t source_, target_;
};
}  // namespace candidates

// ---- signature::Signature (signature.hpp:17-391) -----------------------------------
namespace signature {
enum class Algorithm { ViewBased, PowerGraph };
enum class SignatureScope { Data, Query };

template <Algorithm A = Algorithm::PowerGraph, size_t Bits = 4>
class Signature {
  static_assert(A == Algorithm::PowerGraph && Bits == 4, "the driver path uses Signature<PowerGraph, 4>");

 public:
  Signature(Queue& queue, size_t data_nodes, size_t query_nodes) : q_(queue), dn_(data_nodes), qn_(query_nodes) {
    check(sigmo_signature_create(queue.handle(), data_nodes, query_nodes, &h_));
  }
  ~Signature() { sigmo_signature_destroy(h_); }
  Signature(const Signature&) = delete;
  Signature& operator=(const Signature&) = delete;
  utils::BatchedEvent generateDataSignatures(DeviceBatchedCSRGraph& g) { return gen(g, SIGMO_SCOPE_DATA); }
  utils::BatchedEvent generateQuerySignatures(DeviceBatchedCSRGraph& g) { return gen(g, SIGMO_SCOPE_QUERY); }
  utils::BatchedEvent refineDataSignatures(DeviceBatchedCSRGraph& g, size_t view_size = 1) {
    return ref(g, SIGMO_SCOPE_DATA, view_size);
  }
  utils::BatchedEvent refineQuerySignatures(DeviceBatchedCSRGraph& g, size_t view_size = 1) {
    return ref(g, SIGMO_SCOPE_QUERY, view_size);
  }
  size_t getDataSignatureAllocationSize() const { return size(SIGMO_SCOPE_DATA); }
  size_t getQuerySignatureAllocationSize() const { return size(SIGMO_SCOPE_QUERY); }
  size_t getMaxLabels() const { return 64 / Bits; }
  std::vector<uint64_t> getDataSignatures() const { return download(SIGMO_SCOPE_DATA, dn_); }
  std::vector<uint64_t> getQuerySignatures() const { return download(SIGMO_SCOPE_QUERY, qn_); }
  sigmo_signature_t handle() const { return h_; }

 private:
  utils::BatchedEvent gen(DeviceBatchedCSRGraph& g, int scope) {
    check(sigmo_signature_generate(h_, g.handle, scope));
    return utils::BatchedEvent(q_);
  }
  utils::BatchedEvent ref(DeviceBatchedCSRGraph& g, int scope, size_t view) {
    check(sigmo_signature_refine(h_, g.handle, scope, static_cast<uint32_t>(view)));
    return utils::BatchedEvent(q_);
  }
  size_t size(int scope) const {
    uint64_t b = 0;
    check(sigmo_signature_alloc_size(h_, scope, &b));
    return b;
  }
  std::vector<uint64_t> download(int scope, size_t n) const {
    std::vector<uint64_t> v(n);
    check(sigmo_signature_download(h_, scope, v.data(), n));
    return v;
  }
  Queue& q_;
  sigmo_signature_t h_ = nullptr;
  size_t dn_, qn_;
};
}  // namespace signature

// ---- isomorphism (isomorphism.hpp, gmcr.hpp) ----------------------------------------
namespace isomorphism {
namespace filter {
template <CandidatesDomain D = CandidatesDomain::Query>
utils::BatchedEvent filterCandidates(Queue& queue, DeviceBatchedCSRGraph& query_graph, DeviceBatchedCSRGraph& data_graph,
                                     signature::Signature<>& signatures, candidates::Candidates& candidates) {
  static_assert(D == CandidatesDomain::Query, "the query-major candidate domain is the driver's");
  check(sigmo_filter_candidates(queue.handle(), query_graph.handle, data_graph.handle, signatures.handle(),
                                candidates.handle()));
  return utils::BatchedEvent(queue);
}
template <CandidatesDomain D = CandidatesDomain::Query>
utils::BatchedEvent refineCandidates(Queue& queue, DeviceBatchedCSRGraph& query_graph, DeviceBatchedCSRGraph& data_graph,
                                     signature::Signature<>& signatures, candidates::Candidates& candidates) {
  static_assert(D == CandidatesDomain::Query, "the query-major candidate domain is the driver's");
  check(sigmo_refine_candidates(queue.handle(), query_graph.handle, data_graph.handle, signatures.handle(),
                                candidates.handle()));
  return utils::BatchedEvent(queue);
}
}  // namespace filter

namespace mapping {
class GMCR {
 public:
  explicit GMCR(Queue& queue) : q_(queue) { check(sigmo_gmcr_create(queue.handle(), &h_)); }
  ~GMCR() { sigmo_gmcr_destroy(h_); }
  GMCR(const GMCR&) = delete;
  GMCR& operator=(const GMCR&) = delete;
  utils::BatchedEvent generateGMCR(DeviceBatchedCSRGraph& query_graphs, DeviceBatchedCSRGraph& data_graphs,
                                   candidates::Candidates& candidates) {
    check(sigmo_gmcr_generate(h_, query_graphs.handle, data_graphs.handle, candidates.handle()));
    num_data_graphs_ = data_graphs.num_graphs;
    return utils::BatchedEvent(q_);
  }
  size_t total_query_indices() const {
    uint64_t t = 0;
    check(sigmo_gmcr_total(h_, &t));
    return t;
  }
  // data_graph_offsets [D_g + 1] and query_graph_indices [total] on the host.
  std::pair<std::vector<uint32_t>, std::vector<uint32_t>> getGMCR() const {
    std::vector<uint32_t> off(num_data_graphs_ + 1), idx(total_query_indices());
    check(sigmo_gmcr_download(h_, off.data(), off.size(), idx.data(), idx.size()));
    return {off, idx};
  }
  sigmo_gmcr_t handle() const { return h_; }

 private:
  Queue& q_;
  sigmo_gmcr_t h_ = nullptr;
  uint32_t num_data_graphs_ = 0;
};
}  // namespace mapping

namespace join {
// joinCandidates (isomorphism.hpp:270-381): *num_matches += matches.
inline utils::BatchedEvent joinCandidates(Queue& queue, DeviceBatchedCSRGraph& query_graphs, DeviceBatchedCSRGraph& data_graphs,
                                          candidates::Candidates& candidates, mapping::GMCR& gmcr, size_t* num_matches,
                                          bool find_first = true) {
  uint64_t acc = *num_matches;
  check(sigmo_join_candidates(queue.handle(), query_graphs.handle, data_graphs.handle, candidates.handle(), gmcr.handle(),
                              &acc, find_first ? 1 : 0, nullptr));
  *num_matches = static_cast<size_t>(acc);
  return utils::BatchedEvent(queue);
}

// joinWildcardCandidates (isomorphism.hpp:435-560): bond-label-aware join.
inline utils::BatchedEvent joinWildcardCandidates(Queue& queue, DeviceBatchedCSRGraph& query_graphs,
                                                  DeviceBatchedCSRGraph& data_graphs, candidates::Candidates& candidates,
                                                  mapping::GMCR& gmcr, size_t* num_matches, bool find_first = true) {
  uint64_t acc = *num_matches;
  check(sigmo_join_wildcard_candidates(queue.handle(), query_graphs.handle, data_graphs.handle, candidates.handle(),
                                       gmcr.handle(), &acc, find_first ? 1 : 0, nullptr));
  *num_matches = static_cast<size_t>(acc);
  return utils::BatchedEvent(queue);
}
}  // namespace join
}  // namespace isomorphism

}  // namespace sigmo
