// SIGMo hot-path oracle: a CPU restatement of the reference's batched
// subgraph-isomorphism pipeline.  TEST INFRASTRUCTURE ONLY: it is linked by the
// tests, by __graft_entry__.smoke() and by bench.py's CPU-baseline arm as the
// checker / CPU baseline, never by the product library.
//
// Every function cites the reference file:line it restates (paths are relative
// to the SIGMo project root).  The reference contains C++ undefined behaviour
// (over-wide shifts, a u8-truncated bitset index, a 30-entry DFS stack) whose
// results differ between the NVIDIA PTX target the reference was written for
// and a host x86 target, so every function takes a semantics profile:
//
//   ORC_REF_PTX (0)  shift count >= width gives 0 (PTX shl/shr clamp).  Default
//                    parity contract.
//   ORC_REF_X86 (1)  shift count is masked to the register width (x86 shl/shr).
//   ORC_EXACT   (2)  the mathematically intended semantics: exact sets of any
//                    size (<= 256 vertices per graph), correct range masks, an
//                    injective DFS with clean backtracking.
//
// Pinning: the reference's own hot-path code (library/include/*.hpp) is built
// for the host by oracle/ref_build.py (g++ with the SYCL stand-in
// oracle/sycl_host) and run on seeded inputs; its signatures and candidate
// bitsets after the filter and after every refinement, its GMCR and its
// find-all / find-first totals equal this oracle's ORC_REF_X86 profile
// (tests/test_ref_cpu.py, against the live build and against the committed
// outputs tests/golden/ref_golden.json).  ORC_REF_PTX shares every line with
// ORC_REF_X86 except the three shift helpers below (shl64_one, shl32, shr32);
// ORC_EXACT takes its own branches (exact sets and range masks, an injective
// DFS) and is checked against a brute-force embedding count.  The reference's own
// known-answer tests (library/test/candidates.cpp:13-32,119-143,
// library/test/graphs.cpp:59-120, library/test/filter.cpp:14-68) are checked
// too (tests/test_oracle_cpu.py).

// Build: oracle/Makefile -> oracle/liboracle_sigmo.so (g++ -O3 -fopenmp).

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

enum { ORC_REF_PTX = 0, ORC_REF_X86 = 1, ORC_EXACT = 2 };

// Batched CSR with global vertex ids, exactly the arrays createDeviceCSRGraph
// builds (library/include/graph.hpp:255-314).
typedef struct {
  uint32_t num_graphs;
  uint64_t total_nodes;
  uint64_t total_edges;
  const uint32_t* graph_offsets;  // [num_graphs + 1]
  const uint32_t* row_offsets;    // [total_nodes + 1]
  const uint32_t* column_indices; // [total_edges]
  const uint8_t* node_labels;     // [total_nodes]
} orc_graph;

}  // extern "C"

namespace {

constexpr uint8_t kWildcard = 255;  // types::WILDCARD_NODE, library/include/types.hpp:23
constexpr int kExactWords = 4;      // exact-profile local sets: up to 256 vertices

// ---- shift semantics ------------------------------------------------------
inline uint64_t shl64_one(uint32_t count, int prof) {
  if (prof == ORC_REF_X86) return 1ull << (count & 63u);
  return count >= 64u ? 0ull : (1ull << count);
}
inline uint32_t shl32(uint32_t v, uint32_t count, int prof) {
  if (prof == ORC_REF_X86) return v << (count & 31u);
  return count >= 32u ? 0u : (v << count);
}
inline uint32_t shr32(uint32_t v, uint32_t count, int prof) {
  if (prof == ORC_REF_X86) return v >> (count & 31u);
  return count >= 32u ? 0u : (v >> count);
}

// ---- utils::detail::Bitset<uint64_t> (library/include/utils.hpp:64-96) ----
// The index parameter is uint8_t; (idx - offset) is computed in unsigned int.
struct RefBitset {
  uint64_t data = 0;
  uint32_t offset = 0;
  int prof = ORC_REF_PTX;
  uint32_t count_of(uint32_t idx) const { return static_cast<uint32_t>(static_cast<uint8_t>(idx)) - offset; }
  void set(uint32_t idx) { data |= shl64_one(count_of(idx), prof); }
  void unset(uint32_t idx) { data &= ~shl64_one(count_of(idx), prof); }
  bool get(uint32_t idx) const { return (data & shl64_one(count_of(idx), prof)) != 0; }
  // getSetBit (utils.hpp:85-95): idx-th set bit via repeated ctz; offset is 0
  // at every call site on the driver path (signature BFS).
  uint32_t getSetBit(uint32_t idx) const {
    uint8_t k = static_cast<uint8_t>(static_cast<uint8_t>(idx) - static_cast<uint8_t>(offset));
    uint64_t tmp = data;
    uint32_t ret = 0xFFFFu;
    for (int c = 0; c <= k; ++c) {
      ret = tmp ? static_cast<uint32_t>(__builtin_ctzll(tmp)) : 64u;
      tmp &= ~shl64_one(ret, prof);
    }
    return ret & 0xFFFFu;
  }
};

// ---- Signature<PowerGraph,4>::SignatureDevice (signature.hpp:23-54) --------
inline uint32_t sig_get(uint64_t s, uint32_t label) {
  label &= 0xFFu;
  if (label < 16u) return static_cast<uint32_t>((s >> (label * 4u)) & 0xFu);
  return 0;
}
inline uint64_t sig_set(uint64_t s, uint32_t label, uint32_t count) {
  label &= 0xFFu;
  count &= 0xFFu;
  if (label < 16u && count < 16u) {
    s &= ~(0xFull << (label * 4u));
    s |= static_cast<uint64_t>(count) << (label * 4u);
  }
  return s;
}
inline uint64_t sig_increment(uint64_t s, uint32_t label, uint32_t add = 1) {
  label &= 0xFFu;
  if (label < 16u) {
    uint32_t c = sig_get(s, label);
    if (c < 15u) s = sig_set(s, label, static_cast<uint8_t>(c + static_cast<uint8_t>(add)));
  }
  return s;
}

// DeviceBatchedCSRGraph::getGraphID (graph.hpp:100-111)
inline uint32_t graph_id_of(const orc_graph* g, uint32_t node) {
  size_t lo = 0, hi = g->num_graphs;
  while (lo < hi) {
    size_t mid = lo + (hi - lo) / 2;
    if (node >= g->graph_offsets[mid]) lo = mid + 1;
    else hi = mid;
  }
  return lo > 0 ? static_cast<uint32_t>(lo - 1) : 0xFFFFFFFFu;
}

// DeviceBatchedCSRGraph::isNeighbor (graph.hpp:72-77)
inline bool is_neighbor(const orc_graph* g, uint32_t node, uint32_t nb) {
  for (uint32_t i = g->row_offsets[node]; i < g->row_offsets[node + 1]; ++i)
    if (g->column_indices[i] == nb) return true;
  return false;
}

// ---- CandidatesDevice (candidates.hpp:16-162) -----------------------------
struct Cand {
  const uint32_t* bits;
  uint64_t W;  // single_node_size = ceil(target_nodes / 32)
  int prof;

  // Range mask of word i for the range [s, e) (candidates.hpp:91-99).
  uint32_t mask(uint32_t i, uint32_t s, uint32_t e, uint32_t start_idx, uint32_t end_idx) const {
    if (prof == ORC_EXACT) {
      uint32_t lo = std::max<uint32_t>(s, i * 32u), hi = std::min<uint32_t>(e, i * 32u + 32u);
      if (lo >= hi) return 0u;
      uint32_t len = hi - lo;
      uint32_t m = len >= 32u ? 0xFFFFFFFFu : ((1u << len) - 1u);
      return m << (lo - i * 32u);
    }
    uint32_t m = 0xFFFFFFFFu;
    if (start_idx == end_idx - 1) {
      m = shl32(shr32(m, 32u - (e - s), prof), s % 32u, prof);
    } else if (i == start_idx) {
      m = shl32(m, s % 32u, prof);
    } else if (i == end_idx - 1) {
      m = shr32(m, 32u - (e % 32u), prof);
    }
    return m;
  }
  // getCandidatesCount(source, start, end) (candidates.hpp:86-104)
  uint32_t count(uint64_t src, uint32_t s, uint32_t e) const {
    uint32_t c = 0;
    uint32_t start_idx = s / 32u, end_idx = (e + 31u) / 32u;
    for (uint32_t i = start_idx; i < end_idx; ++i)
      c += static_cast<uint32_t>(__builtin_popcount(bits[src * W + i] & mask(i, s, e, start_idx, end_idx)));
    return c;
  }
  // getCandidateAt(source, idx, start, end) (candidates.hpp:132-162)
  uint32_t at(uint64_t src, uint32_t idx, uint32_t s, uint32_t e) const {
    uint32_t c = 0;
    uint32_t start_idx = s / 32u, end_idx = (e + 31u) / 32u;
    for (uint32_t i = start_idx; i < end_idx; ++i) {
      uint32_t blk = bits[src * W + i] & mask(i, s, e, start_idx, end_idx);
      uint32_t bc = static_cast<uint32_t>(__builtin_popcount(blk));
      if (c + bc > idx) {
        while (blk) {
          uint32_t t = static_cast<uint32_t>(__builtin_ctz(blk));
          if (c == idx) return i * 32u + t;
          blk ^= (1u << t);
          ++c;
        }
      } else {
        c += bc;
      }
    }
    return 0xFFFFFFFFu;
  }
};

// Exact-profile local set of up to 256 vertices.
struct WideSet {
  uint64_t w[kExactWords] = {0, 0, 0, 0};
  void set(uint32_t i) { w[i >> 6] |= 1ull << (i & 63u); }
  void unset(uint32_t i) { w[i >> 6] &= ~(1ull << (i & 63u)); }
  bool get(uint32_t i) const { return (w[i >> 6] >> (i & 63u)) & 1ull; }
  bool empty() const { return !(w[0] | w[1] | w[2] | w[3]); }
};

}  // namespace

extern "C" {

// generateCSRSignatures (signature.hpp:125-152): per vertex, +1 (saturating)
// to the counter of each neighbour's label, on top of the current value.
void orc_generate_signatures(const orc_graph* g, uint64_t* sig) {
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < static_cast<int64_t>(g->total_nodes); ++v) {
    uint64_t s = sig[v];
    for (uint32_t i = g->row_offsets[v]; i < g->row_offsets[v + 1]; ++i)
      s = sig_increment(s, g->node_labels[g->column_indices[i]]);
    sig[v] = s;
  }
}

// refineCSRSignatures<PowerGraph> (signature.hpp:336-390).
// reach has `reach_words` u64 per vertex (1 for ref profiles, 4 for exact);
// the reference keeps it as a 16-byte Bitset whose offset word is never read.
// Returns 0, or -1 if a graph exceeds 256 vertices under the exact profile.
int orc_refine_signatures(const orc_graph* g, uint32_t view_size, int prof, uint64_t* sig, uint64_t* reach,
                          uint32_t reach_words) {
  if (prof == ORC_EXACT) {
    for (uint32_t gi = 0; gi < g->num_graphs; ++gi)
      if (g->graph_offsets[gi + 1] - g->graph_offsets[gi] > 64u * kExactWords) return -1;
    if (reach_words < kExactWords) return -1;
  }
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t vv = 0; vv < static_cast<int64_t>(g->total_nodes); ++vv) {
    uint32_t v = static_cast<uint32_t>(vv);
    uint32_t gid = graph_id_of(g, v);
    uint32_t prev = g->graph_offsets[gid];
    uint64_t* old = reach + static_cast<uint64_t>(v) * reach_words;
    if (prof != ORC_EXACT) {
      RefBitset frontier, reachable;
      frontier.prof = reachable.prof = prof;
      uint64_t old_data = old[0];
      frontier.set(v - prev);
      reachable.set(v - prev);
      for (uint32_t it = 0; it < view_size && frontier.data != 0; ++it) {
        RefBitset next;
        next.prof = prof;
        uint32_t fs = static_cast<uint32_t>(__builtin_popcountll(frontier.data));
        for (uint32_t idx = 0; idx < fs; ++idx) {
          uint32_t u = frontier.getSetBit(idx) + prev;
          for (uint32_t i = g->row_offsets[u]; i < g->row_offsets[u + 1]; ++i) {
            uint32_t nb = g->column_indices[i] - prev;
            if (!reachable.get(nb)) {
              reachable.set(nb);
              next.set(nb);
            }
          }
        }
        frontier = next;
      }
      reachable.unset(v - prev);
      reachable.data &= ~old_data;
      uint64_t s = 0;
      uint32_t rs = static_cast<uint32_t>(__builtin_popcountll(reachable.data));
      for (uint32_t idx = 0; idx < rs; ++idx) {
        uint32_t u = reachable.getSetBit(idx) + prev;
        s = sig_increment(s, g->node_labels[u]);
      }
      sig[v] = s;
      old[0] = reachable.data | old_data;
    } else {
      // Exact sets: ball_r(v) \ {v} \ old(v), labels histogrammed, old |= it.
      WideSet frontier, reachable;
      uint32_t lv = v - prev;
      frontier.set(lv);
      reachable.set(lv);
      for (uint32_t it = 0; it < view_size && !frontier.empty(); ++it) {
        WideSet next;
        for (uint32_t b = 0; b < 64u * kExactWords; ++b) {
          if (!frontier.get(b)) continue;
          uint32_t u = b + prev;
          for (uint32_t i = g->row_offsets[u]; i < g->row_offsets[u + 1]; ++i) {
            uint32_t nb = g->column_indices[i] - prev;
            if (!reachable.get(nb)) {
              reachable.set(nb);
              next.set(nb);
            }
          }
        }
        frontier = next;
      }
      reachable.unset(lv);
      uint64_t s = 0;
      for (int k = 0; k < kExactWords; ++k) {
        uint64_t sphere = reachable.w[k] & ~old[k];
        while (sphere) {
          uint32_t b = static_cast<uint32_t>(__builtin_ctzll(sphere));
          sphere &= sphere - 1;
          s = sig_increment(s, g->node_labels[prev + 64u * k + b]);
        }
        old[k] |= reachable.w[k];
      }
      sig[v] = s;
    }
  }
  return 0;
}

// filterCandidates<Query> (isomorphism.hpp:22-62): bit (q, d) is set when the
// labels are equal or the query label is the wildcard.  ORs into `bits`
// (zero-filled by the Candidates constructor, candidates.hpp:165-179).
void orc_filter(const orc_graph* q, const orc_graph* d, uint32_t* bits) {
  const uint64_t W = (d->total_nodes + 31) / 32;
#pragma omp parallel for schedule(static)
  for (int64_t qi = 0; qi < static_cast<int64_t>(q->total_nodes); ++qi) {
    uint8_t ql = q->node_labels[qi];
    uint32_t* row = bits + static_cast<uint64_t>(qi) * W;
    for (uint64_t dn = 0; dn < d->total_nodes; ++dn)
      if (ql == d->node_labels[dn] || ql == kWildcard) row[dn / 32] |= (1u << (dn % 32));
  }
}

// refineCandidates<Query> (isomorphism.hpp:64-127), race-free form: a set bit
// (q, d) survives iff every 4-bit label counter of sig_q is <= that of sig_d.
void orc_refine(const orc_graph* q, const orc_graph* d, const uint64_t* sigq, const uint64_t* sigd, uint32_t* bits) {
  const uint64_t W = (d->total_nodes + 31) / 32;
#pragma omp parallel for schedule(static)
  for (int64_t qi = 0; qi < static_cast<int64_t>(q->total_nodes); ++qi) {
    uint64_t qs = sigq[qi];
    uint32_t* row = bits + static_cast<uint64_t>(qi) * W;
    for (uint64_t w = 0; w < W; ++w) {
      uint32_t word = row[w];
      uint32_t m = word;
      while (m) {
        uint32_t b = static_cast<uint32_t>(__builtin_ctz(m));
        m &= m - 1;
        uint64_t ds = sigd[w * 32 + b];
        bool keep = true;
        for (uint32_t l = 0; l < 16 && keep; ++l) keep = sig_get(qs, l) <= sig_get(ds, l);
        if (!keep) word &= ~(1u << b);
      }
      row[w] = word;
    }
  }
}

// GMCR::generateGMCR (gmcr.hpp:33-128).  A pair (query graph q, data graph g)
// is admitted iff every query vertex has at least one range-masked candidate in
// g.  Queries with <= 1 vertex are skipped in both the count and the fill
// (the reference counts them in kernel 1 but skips them in kernel 3, leaving
// uninitialised slots; that case is out of domain).  Query ids within a
// segment are written in ascending order (the reference's order is
// nondeterministic).  offsets has num_graphs(d)+1 entries.  Returns the total
// number of admitted pairs; indices is filled only if cap >= total.
uint64_t orc_gmcr(const orc_graph* q, const orc_graph* d, const uint32_t* bits, int prof, uint32_t* offsets,
                  uint32_t* indices, uint64_t cap) {
  const uint64_t W = (d->total_nodes + 31) / 32;
  Cand c{bits, W, prof};
  const uint32_t G = d->num_graphs, QG = q->num_graphs;
  std::vector<std::vector<uint32_t>> seg(G);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t gi = 0; gi < static_cast<int64_t>(G); ++gi) {
    uint32_t s = d->graph_offsets[gi], e = d->graph_offsets[gi + 1];
    for (uint32_t qg = 0; qg < QG; ++qg) {
      uint32_t qoff = q->graph_offsets[qg], n = q->graph_offsets[qg + 1] - qoff;
      if (n <= 1) continue;
      bool add = true;
      for (uint32_t i = 0; i < n && add; ++i) add = c.count(qoff + i, s, e) > 0;
      if (add) seg[gi].push_back(qg);
    }
  }
  offsets[0] = 0;
  for (uint32_t gi = 0; gi < G; ++gi) offsets[gi + 1] = offsets[gi] + static_cast<uint32_t>(seg[gi].size());
  uint64_t total = offsets[G];
  if (indices && cap >= total)
    for (uint32_t gi = 0; gi < G; ++gi) std::copy(seg[gi].begin(), seg[gi].end(), indices + offsets[gi]);
  return total;
}

// isValidMapping (isomorphism.hpp:150-168): induced check against every
// earlier depth, in identity order, labels ignored.
static inline bool valid_mapping(uint32_t cand, uint32_t depth, const uint32_t* mapping, const orc_graph* q, uint32_t qoff,
                                 const orc_graph* d) {
  for (uint32_t i = 0; i < depth; ++i)
    if (is_neighbor(q, i + qoff, depth + qoff) != is_neighbor(d, mapping[i], cand)) return false;
  return true;
}

// joinCandidates (isomorphism.hpp:270-381).  One simulated work-group per
// data graph; work-item lid handles segment slots lid, lid+wg, ...; its
// mapping[] array starts zeroed and is carried across the pairs it handles.
// per_pair (nullable) receives the match count of each GMCR slot.
// Returns the total, or UINT64_MAX if a query has more than 64 vertices or
// (exact profile) a data graph has more than 256.
uint64_t orc_join(const orc_graph* q, const orc_graph* d, const uint32_t* bits, const uint32_t* offsets,
                  const uint32_t* indices, int prof, int find_first, uint32_t wg, uint64_t* per_pair) {
  constexpr uint32_t kMaxDepth = 64;
  for (uint32_t qg = 0; qg < q->num_graphs; ++qg)
    if (q->graph_offsets[qg + 1] - q->graph_offsets[qg] > kMaxDepth) return UINT64_MAX;
  if (prof == ORC_EXACT)
    for (uint32_t gi = 0; gi < d->num_graphs; ++gi)
      if (d->graph_offsets[gi + 1] - d->graph_offsets[gi] > 64u * kExactWords) return UINT64_MAX;
  if (wg == 0) wg = 128;
  const uint64_t W = (d->total_nodes + 31) / 32;
  Cand c{bits, W, prof};
  uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 8) reduction(+ : total)
  for (int64_t gi = 0; gi < static_cast<int64_t>(d->num_graphs); ++gi) {
    const uint32_t s = d->graph_offsets[gi], e = d->graph_offsets[gi + 1];
    const uint32_t seg0 = offsets[gi], seglen = offsets[gi + 1] - offsets[gi];
    for (uint32_t lid = 0; lid < wg && lid < seglen; ++lid) {
      uint32_t mapping[kMaxDepth + 1];
      std::memset(mapping, 0, sizeof(mapping));
      for (uint32_t it = lid; it < seglen; it += wg) {
        const uint32_t qg = indices[seg0 + it];
        const uint32_t qoff = q->graph_offsets[qg];
        const uint32_t n = q->graph_offsets[qg + 1] - qoff;
        uint64_t found = 0;
        struct Frame { uint32_t depth; uint64_t idx; } stack[kMaxDepth + 2];
        uint32_t top = 0;
        stack[top++] = {0, 0};
        if (prof != ORC_EXACT) {
          RefBitset visited;
          visited.offset = s;
          visited.prof = prof;
          while (top > 0) {
            Frame fr = stack[top - 1];
            uint32_t qn = fr.depth;
            if (fr.depth == n) {
              ++found;
              --top;
              if (find_first) break;
              continue;
            }
            if (fr.idx >= c.count(qn + qoff, s, e)) {
              --top;
              visited.unset(mapping[qn]);
              if (top == 1) visited.data = 0;
              continue;
            }
            uint32_t cand = c.at(qn + qoff, static_cast<uint32_t>(fr.idx), s, e);
            stack[top - 1].idx++;
            if (visited.get(cand)) continue;
            if (fr.depth == 0 || valid_mapping(cand, fr.depth, mapping, q, qoff, d)) {
              mapping[fr.depth] = cand;
              visited.set(cand);
              stack[top++] = {fr.depth + 1, 0};
            }
          }
        } else {
          // Exact: injective, each placement undone when its frame resumes.
          WideSet used;
          uint32_t placed[kMaxDepth + 1];
          for (uint32_t k = 0; k <= kMaxDepth; ++k) placed[k] = 0xFFFFFFFFu;
          while (top > 0) {
            Frame fr = stack[top - 1];
            uint32_t qn = fr.depth;
            if (fr.depth == n) {
              ++found;
              --top;
              if (find_first) break;
              continue;
            }
            if (placed[qn] != 0xFFFFFFFFu) {  // resuming: undo this depth's last placement
              used.unset(placed[qn] - s);
              placed[qn] = 0xFFFFFFFFu;
            }
            if (fr.idx >= c.count(qn + qoff, s, e)) {
              --top;
              continue;
            }
            uint32_t cand = c.at(qn + qoff, static_cast<uint32_t>(fr.idx), s, e);
            stack[top - 1].idx++;
            if (used.get(cand - s)) continue;
            if (fr.depth == 0 || valid_mapping(cand, fr.depth, mapping, q, qoff, d)) {
              mapping[fr.depth] = cand;
              placed[qn] = cand;
              used.set(cand - s);
              stack[top++] = {fr.depth + 1, 0};
            }
          }
        }
        if (per_pair) per_pair[seg0 + it] = found;
        total += found;
      }
    }
  }
  return total;
}

// Closed form of the ref-ptx join for data graphs whose first global vertex is
// >= 256: there the visited bitset's shift count is always >= 64, so the DFS
// counts every tuple (d_0..d_{n-1}) of range-masked candidates with
// adjQ(i,j) == adjD(d_i,d_j) for all i < j (non-adjacent query vertices may
// share a data vertex).  Independent brute-force recursion, used only to
// cross-check orc_join.  Returns per-slot counts like orc_join.
uint64_t orc_join_closed_form(const orc_graph* q, const orc_graph* d, const uint32_t* bits, const uint32_t* offsets,
                              const uint32_t* indices, int find_first, uint64_t* per_pair) {
  const uint64_t W = (d->total_nodes + 31) / 32;
  Cand c{bits, W, ORC_REF_PTX};
  uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 8) reduction(+ : total)
  for (int64_t gi = 0; gi < static_cast<int64_t>(d->num_graphs); ++gi) {
    const uint32_t s = d->graph_offsets[gi], e = d->graph_offsets[gi + 1];
    for (uint32_t slot = offsets[gi]; slot < offsets[gi + 1]; ++slot) {
      const uint32_t qg = indices[slot];
      const uint32_t qoff = q->graph_offsets[qg], n = q->graph_offsets[qg + 1] - qoff;
      std::vector<std::vector<uint32_t>> cands(n);
      for (uint32_t j = 0; j < n; ++j) {
        uint32_t k = c.count(qoff + j, s, e);
        for (uint32_t t = 0; t < k; ++t) cands[j].push_back(c.at(qoff + j, t, s, e));
      }
      std::vector<uint32_t> m(n);
      uint64_t cnt = 0;
      bool stop = false;
      // iterative recursion over depth
      std::vector<size_t> pos(n + 1, 0);
      uint32_t depth = 0;
      while (!stop) {
        if (depth == n) {
          ++cnt;
          if (find_first) break;
          --depth;
          continue;
        }
        if (pos[depth] >= cands[depth].size()) {
          pos[depth] = 0;
          if (depth == 0) break;
          --depth;
          continue;
        }
        uint32_t x = cands[depth][pos[depth]++];
        bool ok = true;
        for (uint32_t i = 0; i < depth && ok; ++i)
          ok = is_neighbor(q, qoff + i, qoff + depth) == is_neighbor(d, m[i], x);
        if (ok) {
          m[depth] = x;
          ++depth;
          pos[depth] = 0;
        }
      }
      if (per_pair) per_pair[slot] = cnt;
      total += cnt;
    }
  }
  return total;
}

// getEdgeLabel (graph.hpp:88-93): label of the CSR entry node -> nb, or 255
// (label_t(-1)) when there is none.
static inline uint8_t edge_label(const orc_graph* g, const uint8_t* el, uint32_t node, uint32_t nb) {
  for (uint32_t i = g->row_offsets[node]; i < g->row_offsets[node + 1]; ++i)
    if (g->column_indices[i] == nb) return el[i];
  return 0xFFu;
}

// defineMatchingOrder + isValidMapping + joinWildcardCandidates
// (isomorphism.hpp:383-560).  A work-group of `wg` items per data graph is cut
// into sub-groups of 32; sub-group sg takes GMCR segment slots sg, sg + wg/32,
// ...  For a slot, the matching order starts with the query vertex (among the
// first 32) with the most range-masked candidates (the highest such id; the
// reduce over the sub-group), then the others in identity order.  Lane l of
// the sub-group runs one DFS per starting candidate l, l + 32, ... of that
// root: frames {depth, next index} from depth 1, the uint8-indexed `visited`
// bitset of the driver's join (cleared and re-seeded with the root whenever
// the DFS returns to depth 1), and isValidMapping, which also requires equal
// bond labels on query edges.  find_first ends a lane's DFS at its first
// match, so the count is then the number of starting candidates that
// extend.  mapping[] (indexed by query vertex) starts zeroed per work-item
// and carries over between its DFS runs.  EXACT: injective with clean
// backtracking.  per_pair[slot] = the slot's matches over all its lanes.
// Returns the total, or UINT64_MAX outside the supported domain.
uint64_t orc_join_wildcard(const orc_graph* q, const uint8_t* qel, const orc_graph* d, const uint8_t* del, const uint32_t* bits,
                           const uint32_t* offsets, const uint32_t* indices, int prof, int find_first, uint32_t wg,
                           uint64_t* per_pair) {
  constexpr uint32_t kMaxDepth = 64, kSub = 32;
  for (uint32_t qg = 0; qg < q->num_graphs; ++qg)
    if (q->graph_offsets[qg + 1] - q->graph_offsets[qg] > kMaxDepth) return UINT64_MAX;
  if (prof == ORC_EXACT)
    for (uint32_t gi = 0; gi < d->num_graphs; ++gi)
      if (d->graph_offsets[gi + 1] - d->graph_offsets[gi] > 64u * kExactWords) return UINT64_MAX;
  if (wg == 0) wg = 128;
  const uint32_t nsg = std::max<uint32_t>(1u, wg / kSub);
  const uint64_t W = (d->total_nodes + 31) / 32;
  Cand c{bits, W, prof};
  if (per_pair) std::memset(per_pair, 0, sizeof(uint64_t) * offsets[d->num_graphs]);
  uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : total)
  for (int64_t gi = 0; gi < static_cast<int64_t>(d->num_graphs); ++gi) {
    const uint32_t s = d->graph_offsets[gi], e = d->graph_offsets[gi + 1];
    const uint32_t seg0 = offsets[gi], seglen = offsets[gi + 1] - offsets[gi];
    for (uint32_t sg = 0; sg < nsg; ++sg) {
      for (uint32_t lane = 0; lane < kSub; ++lane) {
        uint32_t mapping[kMaxDepth];
        std::memset(mapping, 0, sizeof(mapping));
        for (uint32_t it = sg; it < seglen; it += nsg) {
          const uint32_t qg = indices[seg0 + it];
          const uint32_t qoff = q->graph_offsets[qg];
          const uint32_t n = q->graph_offsets[qg + 1] - qoff;
          // defineMatchingOrder (isomorphism.hpp:383-408)
          uint32_t max_c = 0;
          int root = -1;
          const uint32_t lanes = std::min<uint32_t>(n, kSub);
          for (uint32_t i = 0; i < lanes; ++i) max_c = std::max(max_c, c.count(qoff + i, s, e));
          for (uint32_t i = 0; i < lanes; ++i)
            if (c.count(qoff + i, s, e) == max_c) root = static_cast<int>(i);
          uint32_t order[kMaxDepth];
          order[0] = static_cast<uint32_t>(root);
          for (uint32_t i = 0, j = 1; i < n; ++i)
            if (static_cast<int>(i) != root) order[j++] = i;
          auto valid = [&](uint32_t cand, uint32_t depth) {
            for (uint32_t i = 0; i < depth; ++i) {
              const bool qa = is_neighbor(q, order[i] + qoff, order[depth] + qoff);
              if (qa != is_neighbor(d, mapping[order[i]], cand)) return false;
              if (qa && edge_label(d, del, mapping[order[i]], cand) != edge_label(q, qel, order[i] + qoff, order[depth] + qoff))
                return false;
            }
            return true;
          };
          uint64_t found = 0;
          for (uint32_t sc = lane; sc < max_c; sc += kSub) {
            struct Frame { uint32_t depth, idx; } stack[kMaxDepth + 2];
            uint32_t top = 0;
            const uint32_t r = order[0];
            mapping[r] = c.at(qoff + r, sc, s, e);
            stack[top++] = {1, 0};
            if (prof != ORC_EXACT) {
              RefBitset visited;
              visited.offset = s;
              visited.prof = prof;
              visited.set(mapping[r]);
              while (top > 0) {
                const Frame fr = stack[top - 1];
                if (fr.depth == n) {
                  ++found;
                  --top;
                  if (find_first) break;
                  continue;
                }
                const uint32_t qn = order[fr.depth];
                if (fr.idx >= c.count(qn + qoff, s, e)) {
                  --top;
                  visited.unset(mapping[qn]);
                  if (top == 1) {
                    visited.data = 0;
                    visited.set(mapping[r]);
                  }
                  continue;
                }
                const uint32_t cand = c.at(qn + qoff, fr.idx, s, e);
                stack[top - 1].idx++;
                if (visited.get(cand)) continue;
                if (valid(cand, fr.depth)) {
                  mapping[qn] = cand;
                  visited.set(cand);
                  stack[top++] = {fr.depth + 1, 0};
                }
              }
            } else {
              WideSet used;
              uint32_t placed[kMaxDepth + 1];
              for (uint32_t k = 0; k <= kMaxDepth; ++k) placed[k] = 0xFFFFFFFFu;
              used.set(mapping[r] - s);
              while (top > 0) {
                const Frame fr = stack[top - 1];
                if (fr.depth == n) {
                  ++found;
                  --top;
                  if (find_first) break;
                  continue;
                }
                if (placed[fr.depth] != 0xFFFFFFFFu) {  // resuming: undo this depth's last placement
                  used.unset(placed[fr.depth] - s);
                  placed[fr.depth] = 0xFFFFFFFFu;
                }
                const uint32_t qn = order[fr.depth];
                if (fr.idx >= c.count(qn + qoff, s, e)) {
                  --top;
                  continue;
                }
                const uint32_t cand = c.at(qn + qoff, fr.idx, s, e);
                stack[top - 1].idx++;
                if (used.get(cand - s)) continue;
                if (valid(cand, fr.depth)) {
                  mapping[qn] = cand;
                  placed[fr.depth] = cand;
                  used.set(cand - s);
                  stack[top++] = {fr.depth + 1, 0};
                }
              }
            }
          }
          if (per_pair) per_pair[seg0 + it] += found;
          total += found;
        }
      }
    }
  }
  return total;
}

// SignatureDevice methods, exported for the reference's signature KAT
// (library/test/candidates.cpp:13-32).
uint64_t orc_sig_set(uint64_t s, uint32_t label, uint32_t count) { return sig_set(s, label, count); }
uint32_t orc_sig_get(uint64_t s, uint32_t label) { return sig_get(s, label); }
uint64_t orc_sig_increment(uint64_t s, uint32_t label, uint32_t add) { return sig_increment(s, label, add); }

// Order-independent digest of a dense [rows][W] candidate bitset, the value
// the library's sigmo_candidates_digest returns for the same bits:
//   sum_q mix64(h_q + q*K2),  h_q = sum_w mix64(word ^ (w*K1))  (mod 2^64).
// Not a reference function: it lets full-size bitsets (gigabytes) be compared
// after every refinement iteration without keeping or moving them.
static inline uint64_t digest_mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

uint64_t orc_digest(const uint32_t* bits, uint64_t rows, uint64_t W) {
  const uint64_t K1 = 0x9E3779B97F4A7C15ull, K2 = 0xC2B2AE3D27D4EB4Full;
  uint64_t total = 0;
#pragma omp parallel for schedule(static) reduction(+ : total)
  for (int64_t r = 0; r < static_cast<int64_t>(rows); ++r) {
    const uint32_t* row = bits + static_cast<uint64_t>(r) * W;
    uint64_t h = 0;
    for (uint64_t w = 0; w < W; ++w) h += digest_mix64(static_cast<uint64_t>(row[w]) ^ (w * K1));
    total += digest_mix64(h + static_cast<uint64_t>(r) * K2);
  }
  return total;
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

}  // extern "C"
