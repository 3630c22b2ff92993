// sigmo — command-line driver over the sigmo_b200 C++ API.  Same flags and
// report lines as the reference's single-GPU driver (library/src/sigmo.cpp:
// 11-220, flags library/src/utils.hpp:41-87), so its log parser
// (scripts/utils/output_analyzer.py) reads this output unchanged.  Extra
// flags: --profile ref-ptx|exact, --batched (whole pipeline in one call).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <locale>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/sigmo/sigmo.hpp"

namespace {

struct Args {
  bool print_candidates = false, skip_join = false, query_data = false, find_all = false, skip_print_candidates = false;
  bool batched = false;
  int refinement_steps = 0;
  std::string query_file, data_file, candidates_domain = "query", profile = "ref-ptx";
  size_t multiply_factor_query = 1, multiply_factor_data = 1;
  size_t max_data_graphs = 1000000, max_query_graphs = 1000;
  size_t join_wg = 128, filter_wg = 512;
  bool filter_active = false;
  size_t filter_min = static_cast<size_t>(-1), filter_max = 0;
};

void usage(const char* argv0) {
  std::cout << "Usage: " << argv0 << " -Q query.dat -D data.dat [options]\n"
            << "  -p, --print-candidates       print the number of candidates of each query vertex (stderr)\n"
            << "  -i, --iterations N           refinement iterations\n"
            << "  -Q FILE / -D FILE            query / data graph files\n"
            << "  -c, --candidates-domain S    query (data is not supported)\n"
            << "  -m, --multiply K             replicate queries and data K times\n"
            << "  -d, --mul-data K / -q, --mul-query K\n"
            << "      --skip-join              stop after the filter\n"
            << "      --find-all               count all matches (default: first match per pair)\n"
            << "      --query-filter MIN[:MAX] keep queries with MIN..MAX vertices\n"
            << "      --skip-candidates-analysis\n"
            << "      --max-data-graphs N / --max-query-graphs N\n"
            << "      --join-work-group N / --filter-work-group N\n"
            << "      --profile ref-ptx|exact  semantics profile (default ref-ptx)\n"
            << "      --batched                run the fused batched form\n"
            << "  -h, --help\n";
}

Args parse(int argc, char** argv) {
  Args a;
  auto need = [&](int& i) -> std::string {
    if (i + 1 >= argc) throw std::runtime_error(std::string("missing value for ") + argv[i]);
    return argv[++i];
  };
  bool haveQ = false, haveD = false;
  for (int i = 1; i < argc; ++i) {
    std::string s = argv[i];
    std::string val;
    auto eq = s.find('=');
    if (s.rfind("--", 0) == 0 && eq != std::string::npos) {
      val = s.substr(eq + 1);
      s = s.substr(0, eq);
    }
    auto get = [&]() { return val.empty() ? need(i) : val; };
    if (s == "-h" || s == "--help") {
      usage(argv[0]);
      std::exit(0);
    } else if (s == "-p" || s == "--print-candidates") a.print_candidates = true;
    else if (s == "-i" || s == "--iterations") a.refinement_steps = std::stoi(get());
    else if (s == "-Q") { a.query_file = get(); haveQ = true; }
    else if (s == "-D") { a.data_file = get(); haveD = true; }
    else if (s == "-c" || s == "--candidates-domain") a.candidates_domain = get();
    else if (s == "-m" || s == "--multiply") a.multiply_factor_data = a.multiply_factor_query = std::stoul(get());
    else if (s == "-d" || s == "--mul-data") a.multiply_factor_data = std::stoul(get());
    else if (s == "-q" || s == "--mul-query") a.multiply_factor_query = std::stoul(get());
    else if (s == "--skip-join") a.skip_join = true;
    else if (s == "--find-all") a.find_all = true;
    else if (s == "--skip-candidates-analysis") a.skip_print_candidates = true;
    else if (s == "--max-data-graphs") a.max_data_graphs = std::stoul(get());
    else if (s == "--max-query-graphs") a.max_query_graphs = std::stoul(get());
    else if (s == "--join-work-group") a.join_wg = std::stoul(get());
    else if (s == "--filter-work-group") a.filter_wg = std::stoul(get());
    else if (s == "--profile") a.profile = get();
    else if (s == "--batched") a.batched = true;
    else if (s == "--query-filter") {
      std::string f = get();
      a.filter_active = true;
      auto c = f.find(':');
      if (c != std::string::npos) {
        a.filter_min = std::stoul(f.substr(0, c));
        a.filter_max = std::stoul(f.substr(c + 1));
      } else {
        a.filter_min = std::stoul(f);
      }
    } else {
      throw std::runtime_error("unknown option " + s);
    }
  }
  if (haveQ && haveD) a.query_data = true;
  else if (haveQ || haveD) throw std::runtime_error("Both query and data files must be provided");
  return a;
}

// formatNumber (library/src/utils.hpp:127-138): '.' thousands separator.
std::string formatNumber(size_t n) {
  std::string s = std::to_string(n), out;
  int c = 0;
  for (auto it = s.rbegin(); it != s.rend(); ++it) {
    if (c && c % 3 == 0) out.push_back('.');
    out.push_back(*it);
    ++c;
  }
  return std::string(out.rbegin(), out.rend());
}

// getBytesSize (library/src/utils.hpp:140-157)
std::string getBytesSize(size_t num_bytes, bool round = true) {
  double bytes = static_cast<double>(num_bytes);
  std::string unit = "B";
  if (num_bytes >= 1024ull * 1024 * 1024) {
    bytes /= 1024.0 * 1024 * 1024;
    unit = "GB";
  } else if (num_bytes >= 1024 * 1024) {
    bytes /= 1024.0 * 1024;
    unit = "MB";
  } else if (num_bytes >= 1024) {
    bytes /= 1024;
    unit = "KB";
  }
  if (round) return std::to_string(static_cast<int>(std::lround(bytes))) + " " + unit;
  return std::to_string(bytes) + " " + unit;
}

using Clock = std::chrono::high_resolution_clock;
long ms(std::chrono::duration<double> d) { return static_cast<long>(std::chrono::duration_cast<std::chrono::milliseconds>(d).count()); }

}  // namespace

int main(int argc, char** argv) try {
  Args args = parse(argc, argv);
  if (!args.query_data) throw std::runtime_error("Specify input data");
  if (args.candidates_domain != "query") throw std::runtime_error("only the query candidates domain is supported");
  sigmo::Profile prof = args.profile == "exact" ? sigmo::Profile::Exact : sigmo::Profile::RefPtx;
  sigmo::Queue queue(0, prof, static_cast<uint32_t>(args.join_wg), static_cast<uint32_t>(args.filter_wg));

  auto query_graphs = sigmo::io::loadCSRGraphsFromFile(args.query_file);
  auto data_graphs = sigmo::io::loadCSRGraphsFromFile(args.data_file);
  if (args.filter_active) {
    query_graphs.erase(std::remove_if(query_graphs.begin(), query_graphs.end(),
                                      [&](const sigmo::CSRGraph& g) {
                                        return g.getNumNodes() > args.filter_max || g.getNumNodes() < args.filter_min;
                                      }),
                       query_graphs.end());
  }
  const size_t nq = query_graphs.size(), nd = data_graphs.size();
  for (size_t i = 1; i < args.multiply_factor_query; ++i) query_graphs.insert(query_graphs.end(), query_graphs.begin(), query_graphs.begin() + nq);
  for (size_t i = 1; i < args.multiply_factor_data; ++i) data_graphs.insert(data_graphs.end(), data_graphs.begin(), data_graphs.begin() + nd);
  if (query_graphs.size() > args.max_query_graphs) query_graphs.resize(args.max_query_graphs, query_graphs.front());
  if (data_graphs.size() > args.max_data_graphs) data_graphs.resize(args.max_data_graphs, data_graphs.front());
  auto dq = sigmo::createDeviceCSRGraph(queue, query_graphs);
  auto dd = sigmo::createDeviceCSRGraph(queue, data_graphs);

  const size_t query_nodes = dq.total_nodes, data_nodes = dd.total_nodes;
  std::cout << "------------- Input Data -------------\n";
  std::cout << "Reed data graph and query graph\n";
  std::cout << "# Query Nodes " << query_nodes << "\n";
  std::cout << "# Query Graphs " << dq.num_graphs << "\n";
  std::cout << "# Data Nodes " << data_nodes << "\n";
  std::cout << "# Data Graphs " << dd.num_graphs << "\n";
  std::cout << "------------- Configs -------------\n";
  std::cout << "Filter domain: " << args.candidates_domain << "\n";
  std::cout << "Filter Work Group Size: " << args.filter_wg << "\n";
  std::cout << "Join Work Group Size: " << args.join_wg << "\n";
  std::cout << "Find all: " << (args.find_all ? "Yes" : "No") << "\n";

  auto setup0 = Clock::now();
  std::cout << "------------- Setup Data -------------\n";
  const size_t data_graph_bytes = sigmo::getDeviceGraphAllocSize(dd), query_graph_bytes = sigmo::getDeviceGraphAllocSize(dq);
  std::cout << "Allocated " << getBytesSize(data_graph_bytes) << " for graph data\n";
  std::cout << "Allocated " << getBytesSize(query_graph_bytes) << " for query data\n";
  sigmo::candidates::Candidates candidates{queue, query_nodes, data_nodes};
  const size_t candidates_bytes = candidates.getAllocationSize();
  std::cout << "Allocated " << getBytesSize(candidates_bytes) << " for candidates\n";
  sigmo::signature::Signature<> signatures{queue, data_nodes, query_nodes};
  const size_t dsb = signatures.getDataSignatureAllocationSize(), qsb = signatures.getQuerySignatureAllocationSize();
  std::cout << "Allocated " << getBytesSize(dsb) << " for data signatures\n";
  std::cout << "Allocated " << getBytesSize(qsb) << " for query signatures\n";
  const size_t tmp = std::max(dsb, qsb);
  std::cout << "Allocated " << getBytesSize(tmp) << " for temporary buffer\n";
  auto setup1 = Clock::now();
  std::cout << "Total allocated memory: " << getBytesSize(dsb + qsb + candidates_bytes + tmp + data_graph_bytes + query_graph_bytes, false)
            << " out of " << getBytesSize(queue.global_mem_size()) << " available on " << queue.device_name() << "\n";

  std::vector<std::chrono::duration<double>> dsig, qsig, filt;
  std::chrono::duration<double> join_time{0};
  size_t num_matches = 0;
  std::cout << "------------- Runtime Filter Phase -------------\n";
  auto filter0 = Clock::now();
  auto mapping0 = filter0, mapping1 = filter0, join0 = filter0, join1 = filter0, filter1 = filter0;
  if (args.batched) {
    sigmo::isomorphism::mapping::GMCR gmcr{queue};
    sigmo_match_result r;
    sigmo::check(sigmo_match_batched(queue.handle(), dq.handle, dd.handle, static_cast<uint32_t>(args.refinement_steps),
                                     args.find_all ? 0 : 1, SIGMO_MATCH_MATERIALIZE_BITSET, candidates.handle(),
                                     gmcr.handle(), &r));
    std::cout << "[*] Batched pipeline: signatures " << std::lround(r.ms_signatures) << " ms, filter " << std::lround(r.ms_filter)
              << " ms, mapping " << std::lround(r.ms_mapping) << " ms, join " << std::lround(r.ms_join) << " ms\n";
    dsig.push_back(std::chrono::duration<double>(r.ms_signatures / 1e3));
    filt.push_back(std::chrono::duration<double>(r.ms_filter / 1e3));
    join_time = std::chrono::duration<double>(r.ms_join / 1e3);
    num_matches = r.total_matches;
    filter1 = mapping0 = mapping1 = join0 = join1 = Clock::now();
  } else {
    std::cout << "[*] Initialization Step:\n";
    auto e1 = signatures.generateDataSignatures(dd);
    queue.wait_and_throw();
    dsig.push_back(e1.getProfilingInfo());
    std::cout << "- Data signatures generated in " << ms(dsig.back()) << " ms\n";
    auto e2 = signatures.generateQuerySignatures(dq);
    queue.wait_and_throw();
    qsig.push_back(e2.getProfilingInfo());
    std::cout << "- Query signatures generated in " << ms(qsig.back()) << " ms\n";
    auto e3 = sigmo::isomorphism::filter::filterCandidates(queue, dq, dd, signatures, candidates);
    queue.wait_and_throw();
    filt.push_back(e3.getProfilingInfo());
    std::cout << "- Candidates filtered in " << ms(filt.back()) << " ms\n";
    for (int step = 1; step <= args.refinement_steps; ++step) {
      std::cout << "[*] Refinement step " << step << ":\n";
      auto a = signatures.refineDataSignatures(dd, step);
      queue.wait_and_throw();
      dsig.push_back(a.getProfilingInfo());
      std::cout << "- Data signatures refined in " << ms(dsig.back()) << " ms\n";
      auto b = signatures.refineQuerySignatures(dq, step);
      queue.wait_and_throw();
      qsig.push_back(b.getProfilingInfo());
      std::cout << "- Query signatures refined in " << ms(qsig.back()) << " ms\n";
      auto c = sigmo::isomorphism::filter::refineCandidates(queue, dq, dd, signatures, candidates);
      queue.wait_and_throw();
      filt.push_back(c.getProfilingInfo());
      std::cout << "- Candidates refined in " << ms(filt.back()) << " ms\n";
    }
    filter1 = Clock::now();
    if (!args.skip_join) {
      std::cout << "[*] Generating DQCR\n";
      mapping0 = Clock::now();
      sigmo::isomorphism::mapping::GMCR gmcr{queue};
      gmcr.generateGMCR(dq, dd, candidates);
      mapping1 = Clock::now();
      std::cout << "[*] Starting Join\n";
      join0 = Clock::now();
      auto je = sigmo::isomorphism::join::joinCandidates(queue, dq, dd, candidates, gmcr, &num_matches, !args.find_all);
      je.wait();
      join_time = je.getProfilingInfo();
      join1 = Clock::now();
    }
  }
  std::cout << "[!] End\n";
  auto sum = [](const std::vector<std::chrono::duration<double>>& v) {
    return std::accumulate(v.begin(), v.end(), std::chrono::duration<double>(0));
  };
  std::cout << "------------- Overall GPU Stats -------------\n";
  const auto tq = sum(qsig), td = sum(dsig), tf = sum(filt);
  std::cout << "Data signature time: " << ms(td) << " ms\n";
  std::cout << "Query signature time: " << ms(tq) << " ms\n";
  std::cout << "Filter time: " << ms(tf) << " ms\n";
  if (args.skip_join) std::cout << "Join time: skipped\n";
  else std::cout << "Join time: " << ms(join_time) << " ms\n";
  std::cout << "Total time: " << ms(td + tf + tq + join_time) << " ms\n";
  std::cout << "------------- Overall Host Stats -------------\n";
  std::cout << "Setup Data time: " << ms(setup1 - setup0) << " ms (not included in total)\n";
  std::cout << "Filter time: " << ms(filter1 - filter0) << " ms\n";
  if (args.skip_join) {
    std::cout << "Mapping time: skipped\n";
    std::cout << "Join time: skipped\n";
  } else {
    std::cout << "Mapping time: " << ms(mapping1 - mapping0) << " ms\n";
    std::cout << "Join time: " << ms(join1 - join0) << " ms\n";
  }
  std::cout << "Total time: " << ms(Clock::now() - setup1) << " ms\n";
  std::cout << "------------- Results -------------\n";
  if (!args.skip_print_candidates) {
    // CandidatesInspector (library/src/utils.hpp:159-178), counts computed on the device
    auto counts = candidates.getCandidatesCounts();
    size_t total = 0, zero = 0;
    for (size_t i = 0; i < counts.size(); ++i) {
      total += counts[i];
      zero += counts[i] == 0;
      if (args.print_candidates) std::cerr << "Node " << i << ": " << counts[i] << "\n";
    }
    std::vector<uint32_t> sorted(counts.begin(), counts.end());
    std::sort(sorted.begin(), sorted.end());
    const size_t avg = counts.empty() ? 0 : total / counts.size();
    const size_t median = sorted.empty() ? 0 : sorted[sorted.size() / 2];
    std::cout << "# Total candidates: " << formatNumber(total) << "\n";
    std::cout << "# Average candidates: " << formatNumber(avg) << "\n";
    std::cout << "# Median candidates: " << formatNumber(median) << "\n";
    std::cout << "# Zero candidates: " << formatNumber(zero) << "\n";
  }
  if (!args.skip_join) std::cout << "# Matches: " << formatNumber(num_matches) << "\n";
  sigmo::destroyDeviceCSRGraph(dd, queue);
  sigmo::destroyDeviceCSRGraph(dq, queue);
  return 0;
} catch (const std::exception& e) {
  std::cerr << "error: " << e.what() << "\n";
  return 1;
}
