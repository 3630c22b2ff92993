// Seeded synthetic molecule and query generator.  SIGMo's benchmark inputs
// (the Ehrlich-Rarey SMARTS set and ZINC, data/README.md) are not available,
// so these graphs stand in for them with the reference's label encoding
// (scripts/smile2graph.py:13-14) and drug-like shapes: max degree 4, 0-3
// rings of 5/6 atoms (aromatic 6-rings), atom mix C 70% N 11% O 12% S 2%
// F 2% Cl 1.5% Br 0.5% P 1%, bonds single/double/triple/aromatic.
//
// Every graph is generated from its own seed (seed, kind, index), so a batch
// is reproducible regardless of how it is split.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.hpp"
#include "host_graphs.hpp"

namespace sigmo_b200 {
namespace {

enum Label : uint8_t { L_N = 0, L_Cl = 1, L_Star = 2, L_Br = 3, L_I = 4, L_P = 5, L_H = 6, L_O = 7, L_C = 8, L_S = 9, L_F = 10 };
enum Bond : uint8_t { B_SINGLE = 1, B_DOUBLE = 2, B_TRIPLE = 3, B_AROMATIC = 4 };

inline uint64_t splitmix64(uint64_t& x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct Rng {
  uint64_t s[4];
  explicit Rng(uint64_t seed) {
    uint64_t x = seed;
    for (auto& w : s) w = splitmix64(x);
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {  // xoshiro256**
    uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
  uint32_t below(uint32_t n) { return n ? static_cast<uint32_t>((next() >> 32) * n >> 32) : 0; }
  uint32_t range(uint32_t lo, uint32_t hi) { return lo + below(hi - lo + 1); }  // inclusive
  double normal() {
    double u1 = std::max(uniform(), 1e-300), u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

uint64_t graph_seed(uint64_t seed, uint64_t stream, uint64_t index) {
  uint64_t x = seed ^ (stream * 0xD1B54A32D192ED03ull);
  splitmix64(x);
  x ^= index * 0x9E3779B97F4A7C15ull;
  return splitmix64(x);
}

struct MolBuilder {
  uint32_t n = 0;
  std::vector<uint8_t> deg, aromatic;
  std::vector<TextEdge> edges;
  std::vector<uint8_t> labels;

  uint32_t add_atom() {
    deg.push_back(0);
    aromatic.push_back(0);
    return n++;
  }
  void bond(uint32_t a, uint32_t b, uint8_t l) {
    edges.push_back({a, b, l});
    deg[a]++;
    deg[b]++;
  }
  // A ring of `size` new atoms; returns first atom id.
  uint32_t ring(uint32_t size, bool arom) {
    uint32_t first = n;
    for (uint32_t i = 0; i < size; ++i) add_atom();
    for (uint32_t i = 0; i < size; ++i) {
      uint32_t a = first + i, b = first + (i + 1) % size;
      bond(a, b, arom ? B_AROMATIC : B_SINGLE);
      if (arom) aromatic[a] = 1;
    }
    return first;
  }
  // A ring fused on the existing bond (a, b): size-2 new atoms a-x1..xk-b.
  void fused_ring(uint32_t a, uint32_t b, uint32_t size, bool arom) {
    uint32_t prev = a;
    for (uint32_t i = 0; i + 2 < size; ++i) {
      uint32_t x = add_atom();
      bond(prev, x, arom ? B_AROMATIC : B_SINGLE);
      if (arom) aromatic[x] = 1;
      prev = x;
    }
    bond(prev, b, arom ? B_AROMATIC : B_SINGLE);
  }
  int pick_open(Rng& r, uint32_t max_deg, uint32_t lo = 0) {
    uint32_t cnt = 0;
    for (uint32_t i = lo; i < n; ++i) cnt += deg[i] < max_deg;
    if (!cnt) return -1;
    uint32_t k = r.below(cnt);
    for (uint32_t i = lo; i < n; ++i)
      if (deg[i] < max_deg && k-- == 0) return static_cast<int>(i);
    return -1;
  }
  uint8_t tree_bond(Rng& r) {
    double u = r.uniform();
    return u < 0.84 ? B_SINGLE : (u < 0.985 ? B_DOUBLE : B_TRIPLE);
  }
  // Grow a tree of `count` atoms hanging off the structure (chain-biased).
  void grow(Rng& r, uint32_t count, double chain_bias) {
    uint32_t last = n ? n - 1 : 0;
    for (uint32_t i = 0; i < count; ++i) {
      if (n == 0) {
        add_atom();
        last = 0;
        continue;
      }
      int at;
      if (r.uniform() < chain_bias && deg[last] < 3) at = static_cast<int>(last);
      else at = pick_open(r, 3);
      if (at < 0) at = pick_open(r, 4);
      if (at < 0) return;  // saturated (cannot happen for trees with max degree 4)
      uint32_t x = add_atom();
      bond(static_cast<uint32_t>(at), x, tree_bond(r));
      last = x;
    }
  }
  // Atom labels chosen per degree so the overall mix is drug-like.
  void assign_labels(Rng& r) {
    labels.assign(n, L_C);
    for (uint32_t i = 0; i < n; ++i) {
      double u = r.uniform();
      uint8_t l = L_C;
      if (aromatic[i]) {
        l = u < 0.86 ? L_C : (u < 0.97 ? L_N : (u < 0.99 ? L_S : L_O));
        if (deg[i] > 3 && l != L_C) l = L_C;
      } else if (deg[i] >= 4) {
        l = u < 0.97 ? L_C : L_S;
      } else if (deg[i] == 3) {
        l = u < 0.78 ? L_C : (u < 0.94 ? L_N : (u < 0.98 ? L_P : L_S));
      } else if (deg[i] == 2) {
        l = u < 0.68 ? L_C : (u < 0.84 ? L_O : (u < 0.96 ? L_N : L_S));
      } else {  // terminal
        l = u < 0.52 ? L_C : (u < 0.76 ? L_O : (u < 0.86 ? L_N : (u < 0.92 ? L_F : (u < 0.965 ? L_Cl : (u < 0.98 ? L_Br : (u < 0.99 ? L_S : L_P))))));
      }
      labels[i] = l;
    }
  }
  void finish(TextGraph* out) {
    out->num_nodes = n;
    out->max_labels = 11;
    out->node_labels = labels;
    out->edges = edges;
  }
};

// kind 0: uniform sizes, 0-3 rings.  kind 1: lognormal sizes, 5% macrocycles
// or fused multi-ring systems.  kind 2: ring-rich (2-6 fused aromatic
// 6-cycles plus carbon chains up to 20 atoms).
void gen_molecule(int kind, uint32_t target, Rng& r, TextGraph* out) {
  MolBuilder m;
  if (target == 0) {
    m.finish(out);
    return;
  }
  if (kind == 2) {
    uint32_t fused = r.range(2, 6);
    uint32_t a = m.ring(6, true);
    uint32_t ra = a, rb = a + 1;
    for (uint32_t k = 1; k < fused && m.n + 4 <= std::max<uint32_t>(target, 10); ++k) {
      uint32_t before = m.n;
      m.fused_ring(ra, rb, 6, true);
      // next fusion on an outer bond of the ring just made
      ra = before + 1;
      rb = before + 2;
      if (rb >= m.n) {
        ra = before;
        rb = before + 1;
      }
    }
    while (m.n < target) {
      uint32_t chain = std::min<uint32_t>(target - m.n, r.range(2, 20));
      int at = m.pick_open(r, 3);
      if (at < 0) break;
      uint32_t prev = static_cast<uint32_t>(at);
      for (uint32_t i = 0; i < chain; ++i) {
        uint32_t x = m.add_atom();
        m.bond(prev, x, B_SINGLE);
        prev = x;
      }
    }
    m.labels.assign(m.n, L_C);
    for (uint32_t i = 0; i < m.n; ++i) {  // mostly carbon, a few heteroatoms
      double u = r.uniform();
      if (!m.aromatic[i] && m.deg[i] <= 2 && u < 0.08) m.labels[i] = u < 0.04 ? L_O : L_N;
      else if (m.aromatic[i] && u < 0.03) m.labels[i] = L_N;
    }
    m.finish(out);
    return;
  }
  bool special = (kind == 1) && r.uniform() < 0.05;
  if (special && target >= 14) {
    if (r.uniform() < 0.5) {  // macrocycle
      uint32_t size = std::min<uint32_t>(target, r.range(12, 24));
      m.ring(size, false);
    } else {  // fused multi-ring system
      uint32_t rings = r.range(3, 5);
      uint32_t a = m.ring(6, true);
      uint32_t ra = a + 2, rb = a + 3;
      for (uint32_t k = 1; k < rings && m.n + 4 <= target; ++k) {
        uint32_t before = m.n;
        uint32_t size = r.uniform() < 0.8 ? 6 : 5;
        m.fused_ring(ra, rb, size, size == 6);
        ra = before;
        rb = before + 1;
      }
    }
  } else {
    double u = r.uniform();
    uint32_t rings = u < 0.22 ? 0 : (u < 0.55 ? 1 : (u < 0.83 ? 2 : 3));
    for (uint32_t k = 0; k < rings; ++k) {
      uint32_t size = r.uniform() < 0.72 ? 6 : 5;
      if (m.n + size > target) break;
      bool arom = size == 6 && r.uniform() < 0.7;
      if (m.n > 0 && r.uniform() < 0.25) {
        // fuse onto a bond of an existing ring atom pair (a, a+1) in a ring
        int fa = -1, fb = -1;
        for (int tries = 0; tries < 8 && fa < 0; ++tries) {
          uint32_t c = r.below(m.n);
          for (const auto& e : m.edges)
            if (e.u == c && m.deg[e.u] <= 2 && m.deg[e.v] <= 2 && (m.aromatic[e.u] || e.label == B_SINGLE)) {
              fa = static_cast<int>(e.u);
              fb = static_cast<int>(e.v);
              break;
            }
        }
        if (fa >= 0) {
          m.fused_ring(static_cast<uint32_t>(fa), static_cast<uint32_t>(fb), size, arom && m.aromatic[fa]);
          continue;
        }
      }
      int at = m.n ? m.pick_open(r, 3) : -1;
      if (m.n && at < 0) break;
      // a linker atom between rings sometimes
      if (at >= 0 && r.uniform() < 0.4 && m.n + size + 1 <= target) {
        uint32_t x = m.add_atom();
        m.bond(static_cast<uint32_t>(at), x, B_SINGLE);
        at = static_cast<int>(x);
      }
      uint32_t first = m.ring(size, arom);
      if (at >= 0) m.bond(static_cast<uint32_t>(at), first + r.below(size), B_SINGLE);
    }
  }
  if (m.n < target) m.grow(r, target - m.n, 0.45);
  m.assign_labels(r);
  m.finish(out);
}

uint32_t sample_size(int kind, uint32_t lo, uint32_t hi, double median, Rng& r) {
  if (hi < lo) std::swap(lo, hi);
  if (kind == 1) {
    double mu = std::log(median > 0 ? median : 22.0), sigma = 0.42;
    for (int t = 0; t < 64; ++t) {
      double x = std::exp(mu + sigma * r.normal());
      uint32_t k = static_cast<uint32_t>(std::lround(x));
      if (k >= lo && k <= hi) return k;
    }
    return std::min(std::max(static_cast<uint32_t>(median), lo), hi);
  }
  return r.range(lo, hi);
}

// Connected induced subgraph of `src` with k vertices, grown from a random
// start by random frontier expansion; vertices renumbered in growth order.
bool induced_subgraph(const TextGraph& src, uint32_t k, Rng& r, TextGraph* out) {
  const uint32_t n = src.num_nodes;
  if (k == 0 || k > n) return false;
  std::vector<std::vector<uint32_t>> adj(n);
  for (const auto& e : src.edges) {
    adj[e.u].push_back(e.v);
    if (e.u != e.v) adj[e.v].push_back(e.u);
  }
  std::vector<int32_t> newid(n, -1);
  std::vector<uint32_t> order;
  std::vector<uint32_t> frontier;
  uint32_t s = r.below(n);
  newid[s] = 0;
  order.push_back(s);
  for (uint32_t v : adj[s]) frontier.push_back(v);
  while (order.size() < k) {
    // drop already-taken entries
    frontier.erase(std::remove_if(frontier.begin(), frontier.end(), [&](uint32_t v) { return newid[v] >= 0; }), frontier.end());
    if (frontier.empty()) return false;
    uint32_t pick = frontier[r.below(static_cast<uint32_t>(frontier.size()))];
    newid[pick] = static_cast<int32_t>(order.size());
    order.push_back(pick);
    for (uint32_t v : adj[pick])
      if (newid[v] < 0) frontier.push_back(v);
  }
  out->num_nodes = k;
  out->max_labels = 11;
  out->node_labels.resize(k);
  out->edges.clear();
  for (uint32_t i = 0; i < k; ++i) out->node_labels[i] = src.node_labels[order[i]];
  for (const auto& e : src.edges) {
    int32_t a = newid[e.u], b = newid[e.v];
    if (a >= 0 && b >= 0) out->edges.push_back({static_cast<uint32_t>(std::min(a, b)), static_cast<uint32_t>(std::max(a, b)), e.label});
  }
  std::sort(out->edges.begin(), out->edges.end(), [](const TextEdge& x, const TextEdge& y) {
    return x.u != y.u ? x.u < y.u : x.v < y.v;
  });
  return true;
}

// Highly automorphic carbon patterns (symmetry stress queries).
void automorphic_query(uint32_t lo, uint32_t hi, Rng& r, TextGraph* out) {
  MolBuilder m;
  uint32_t kind = r.below(5);
  if (kind == 0) {  // benzene-like 6-cycle
    m.ring(6, true);
  } else if (kind == 1) {  // fused bicycle (naphthalene-like)
    m.ring(6, true);
    m.fused_ring(0, 1, 6, true);
  } else if (kind == 2) {  // fused tricycle
    m.ring(6, true);
    m.fused_ring(0, 1, 6, true);
    m.fused_ring(7, 8, 6, true);
  } else if (kind == 3) {  // unlabeled carbon chain
    uint32_t len = r.range(std::max<uint32_t>(lo, 4), std::max<uint32_t>(std::min<uint32_t>(hi, 12), 4));
    m.add_atom();
    for (uint32_t i = 1; i < len; ++i) {
      uint32_t x = m.add_atom();
      m.bond(x - 1, x, B_SINGLE);
    }
  } else {  // branched carbon star
    uint32_t c = m.add_atom();
    uint32_t arms = r.range(3, 4);
    for (uint32_t a = 0; a < arms; ++a) {
      uint32_t prev = c;
      uint32_t len = r.range(1, 2);
      for (uint32_t i = 0; i < len; ++i) {
        uint32_t x = m.add_atom();
        m.bond(prev, x, B_SINGLE);
        prev = x;
      }
    }
  }
  m.labels.assign(m.n, L_C);
  m.finish(out);
}

int emit(const std::vector<TextGraph>& tgs, sigmo_host_graphs* out) {
  std::vector<LocalCSR> csr(tgs.size());
  for (size_t i = 0; i < tgs.size(); ++i) to_csr(tgs[i], &csr[i]);
  return batch_graphs(csr, out);
}

}  // namespace
}  // namespace sigmo_b200

using namespace sigmo_b200;

extern "C" {

int sigmo_generate_molecules(int kind, uint32_t count, uint32_t min_atoms, uint32_t max_atoms, double median,
                             uint64_t seed, sigmo_host_graphs* out) {
  if (!out) return fail(SIGMO_ERR_INVALID, "sigmo_generate_molecules: null output");
  if (kind < 0 || kind > 2) return fail(SIGMO_ERR_INVALID, "sigmo_generate_molecules: kind %d", kind);
  if (max_atoms < min_atoms || max_atoms == 0) return fail(SIGMO_ERR_INVALID, "sigmo_generate_molecules: size range [%u, %u]", min_atoms, max_atoms);
  std::memset(out, 0, sizeof(*out));
  std::vector<TextGraph> tgs(count);
  for (uint32_t i = 0; i < count; ++i) {
    Rng r(graph_seed(seed, 1 + kind, i));
    uint32_t k = sample_size(kind, min_atoms, max_atoms, median, r);
    gen_molecule(kind, k, r, &tgs[i]);
  }
  return emit(tgs, out);
}

int sigmo_generate_queries(int kind, uint32_t count, uint32_t min_atoms, uint32_t max_atoms, uint32_t skew_lo,
                           uint32_t skew_hi, uint64_t seed, sigmo_host_graphs* out) {
  if (!out) return fail(SIGMO_ERR_INVALID, "sigmo_generate_queries: null output");
  if (kind < 0 || kind > 3) return fail(SIGMO_ERR_INVALID, "sigmo_generate_queries: kind %d", kind);
  if (max_atoms < min_atoms || max_atoms == 0) return fail(SIGMO_ERR_INVALID, "sigmo_generate_queries: size range [%u, %u]", min_atoms, max_atoms);
  std::memset(out, 0, sizeof(*out));
  std::vector<TextGraph> tgs(count);
  for (uint32_t i = 0; i < count; ++i) {
    Rng r(graph_seed(seed, 101 + kind, i));
    if (kind == 3) {
      automorphic_query(min_atoms, max_atoms, r, &tgs[i]);
      continue;
    }
    uint32_t k;
    if (skew_lo && skew_hi >= skew_lo && r.uniform() < 0.7) k = r.range(std::max(skew_lo, min_atoms), std::min(skew_hi, max_atoms));
    else k = r.range(min_atoms, max_atoms);
    for (int attempt = 0;; ++attempt) {
      TextGraph src;
      uint32_t srcsize = std::max<uint32_t>(k + r.below(16), 10);
      gen_molecule(kind == 2 ? 2 : 0, srcsize, r, &src);
      if (induced_subgraph(src, k, r, &tgs[i])) break;
      if (attempt > 64) return fail(SIGMO_ERR_DOMAIN, "could not sample a connected %u-vertex query", k);
    }
  }
  return emit(tgs, out);
}

}  // extern "C"
