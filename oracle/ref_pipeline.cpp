// Driver of the reference's own hot-path code on the host CPU — TEST
// INFRASTRUCTURE (built by oracle/ref_build.py into oracle/_ref/, with
// oracle/sycl_host standing in for SYCL).  It follows the stage order of the
// reference's driver (library/src/sigmo.cpp:98-160) through the reference's
// API and writes every intermediate to a dump file that oracle/ref.py reads.
//
//   ref_pipeline <query.dat> <data.dat> <iterations> <join_work_group_size> <out.bin>
//
// Dump records: u32 name length, name, u32 element size, u64 count, data.
//   sig_data_<r>, sig_query_<r>   u64 signatures after the filter (r = 0) and
//                                 after refinement r
//   bits_<r>                      u32 candidate words, [query vertex][words]
//   gmcr_offsets, gmcr_indices    u32 GMCR arrays
//   total_all, total_first        u64 joinCandidates totals (find-all, find-first)
#include <sycl/sycl.hpp>

#include <cstdio>
#include <string>
#include <vector>

#include "sigmo.hpp"

namespace {

struct Dump {
  FILE* f;
  template <typename T>
  void put(const std::string& name, const T* p, uint64_t n) {
    const uint32_t nl = static_cast<uint32_t>(name.size()), es = sizeof(T);
    std::fwrite(&nl, 4, 1, f);
    std::fwrite(name.data(), 1, nl, f);
    std::fwrite(&es, 4, 1, f);
    std::fwrite(&n, 8, 1, f);
    if (n) std::fwrite(p, sizeof(T), n, f);
  }
};

}  // namespace

int main(int argc, char** argv) {
  if (argc != 6) {
    std::fprintf(stderr, "usage: %s query.dat data.dat iterations join_wg out.bin\n", argv[0]);
    return 2;
  }
  const size_t R = std::stoul(argv[3]);
  sigmo::device::deviceOptions.join_work_group_size = std::stoul(argv[4]);
  FILE* f = std::fopen(argv[5], "wb");
  if (!f) return 3;
  Dump dump{f};

  sycl::queue queue{sycl::gpu_selector_v, sycl::property::queue::enable_profiling{}};
  auto query_graphs = sigmo::io::loadCSRGraphsFromFile(argv[1]);
  auto data_graphs = sigmo::io::loadCSRGraphsFromFile(argv[2]);
  auto device_query_graph = sigmo::createDeviceCSRGraph(queue, query_graphs);
  auto device_data_graph = sigmo::createDeviceCSRGraph(queue, data_graphs);
  const size_t query_nodes = device_query_graph.total_nodes, data_nodes = device_data_graph.total_nodes;

  sigmo::candidates::Candidates candidates{queue, query_nodes, data_nodes};
  sigmo::signature::Signature<> signatures{queue, data_nodes, query_nodes};

  auto snapshot = [&](size_t r) {
    const std::string k = std::to_string(r);
    dump.put("sig_data_" + k, reinterpret_cast<const uint64_t*>(signatures.getDeviceDataSignatures()), data_nodes);
    dump.put("sig_query_" + k, reinterpret_cast<const uint64_t*>(signatures.getDeviceQuerySignatures()), query_nodes);
    auto host = candidates.getHostCandidates();
    dump.put("bits_" + k, host.candidates, host.source_nodes * host.single_node_size);
  };

  signatures.generateDataSignatures(device_data_graph);
  queue.wait_and_throw();
  signatures.generateQuerySignatures(device_query_graph);
  queue.wait_and_throw();
  sigmo::isomorphism::filter::filterCandidates(queue, device_query_graph, device_data_graph, signatures, candidates);
  queue.wait_and_throw();
  snapshot(0);
  for (size_t r = 1; r <= R; ++r) {
    signatures.refineDataSignatures(device_data_graph, r);
    queue.wait_and_throw();
    signatures.refineQuerySignatures(device_query_graph, r);
    queue.wait_and_throw();
    sigmo::isomorphism::filter::refineCandidates(queue, device_query_graph, device_data_graph, signatures, candidates);
    queue.wait_and_throw();
    snapshot(r);
  }

  sigmo::isomorphism::mapping::GMCR gmcr{queue};
  gmcr.generateGMCR(device_query_graph, device_data_graph, candidates);
  auto g = gmcr.getGMCRDevice();
  dump.put("gmcr_offsets", g.data_graph_offsets, device_data_graph.num_graphs + 1);
  dump.put("gmcr_indices", g.query_graph_indices, g.total_query_indices);

  for (int find_first = 0; find_first <= 1; ++find_first) {
    size_t* num_matches = sycl::malloc_shared<size_t>(1, queue);
    num_matches[0] = 0;
    auto e = sigmo::isomorphism::join::joinCandidates(queue, device_query_graph, device_data_graph, candidates, gmcr, num_matches,
                                                      find_first != 0);
    e.wait();
    const uint64_t total = num_matches[0];
    dump.put(find_first ? "total_first" : "total_all", &total, 1);
    sycl::free(num_matches, queue);
  }
  std::fclose(f);
  sigmo::destroyDeviceCSRGraph(device_data_graph, queue);
  sigmo::destroyDeviceCSRGraph(device_query_graph, queue);
  return 0;
}
