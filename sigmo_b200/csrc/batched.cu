// The batched form (sigmo_match_batched): signatures for all iterations in
// one BFS, per-graph candidate planes, GMCR from the plane AND-programs, and
// the persistent join, with one host synchronisation (the admitted-pair
// total, as in gmcr.hpp:80) between the launches.  Results are identical to
// the stage-per-launch calls (library/src/sigmo.cpp:98-160).
#include <cuda_runtime.h>

#include <algorithm>
#include <thread>
#include <cstring>
#include <vector>

#include "internal.hpp"

namespace sigmo_b200 {
namespace {

void free_groups(Queue* q, PlaneProgram* pp) {
  for (PlaneGroup& g : pp->groups) {
    dev_free(q, g.spec);
    dev_free(q, g.r_begin);
    dev_free(q, g.row_of);
    dev_free(q, g.prog);
    dev_free(q, g.qc_off);
    dev_free(q, g.qc);
  }
  pp->groups.clear();
}

void free_program(Queue* q, PlaneProgram* pp) {
  free_groups(q, pp);
  dev_free(q, pp->spec);
  dev_free(q, pp->prog_off);
  dev_free(q, pp->prog);
  dev_free(q, pp->cls);
  dev_free(q, pp->r_begin);
  dev_free(q, pp->qc_off);
  dev_free(q, pp->qc);
  dev_free(q, pp->qsig_all);
  pp->qc_off = pp->qc = nullptr;
  *pp = PlaneProgram{};
}

// Threads for host loops over n items: one per 1,024 items, at most 8 and at
// most the machine's hardware threads.
unsigned host_threads(uint64_t n) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  return static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>({n / 1024, 8, hw})));
}
// f(part, begin, end) over `parts` contiguous ranges of [0, n), part 0 on the
// calling thread; parts <= 1 (or `force_serial`) runs inline.
template <class F>
void parallel_ranges(uint64_t n, unsigned parts, F&& f, int force_serial = 0) {
  if (parts <= 1 || force_serial) {
    for (unsigned p = 0; p < parts; ++p) f(p, n * p / parts, n * (p + 1) / parts);
    if (parts == 0) f(0, 0, n);
    return;
  }
  std::vector<std::thread> th;
  th.reserve(parts - 1);
  for (unsigned p = 1; p < parts; ++p) th.emplace_back([&, p] { f(p, n * p / parts, n * (p + 1) / parts); });
  f(0, 0, n / parts);
  for (auto& t : th) t.join();
}

int upload(Queue* q, void** dst, const void* src, size_t bytes) {
  SIGMO_TRY(dev_alloc(q, dst, bytes ? bytes : 4));
  if (bytes) SIGMO_CUDA_TRY(cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, q->stream));
  return SIGMO_OK;
}

}  // namespace

// Builds (or reuses) the plane program of a query batch for R iterations:
// query signatures of iterations 1..R on the device, then on the host the
// distinct labels and (r, l, c) thresholds (the planes), the classes of
// identical (label, signature_1..R) vertices, and each class's program
// (label plane first, then its thresholds).
int build_plane_program(Queue* q, Graph* query, uint32_t R) {
  PlaneProgram& pp = query->pp;
  if (pp.valid && pp.R == R && pp.profile == q->opts.profile) return SIGMO_OK;
  free_program(q, &pp);
  // The program's device work runs on the side stream after the query
  // graph's own creation work only, so a data graph upload queued on the main
  // stream meanwhile overlaps the host work below.
  struct OnSide {
    Queue* q;
    cudaStream_t main;
    ~OnSide() { q->stream = main; }
  } on_side{q, q->stream};
  if (query->ready) SIGMO_CUDA_TRY(cudaStreamWaitEvent(q->side, query->ready, 0));
  q->stream = q->side;
  const uint64_t Qn = query->total_nodes;
  SIGMO_TRY(dev_alloc(q, reinterpret_cast<void**>(&pp.qsig_all), 8ull * (R ? R : 1) * (Qn ? Qn : 1)));
  SIGMO_TRY(launch_sig_all(q, query, R, pp.qsig_all));
  std::vector<uint64_t> sig(static_cast<size_t>(R) * Qn);
  std::vector<uint8_t> lab(Qn);
  if (Qn) {
    if (R) SIGMO_CUDA_TRY(cudaMemcpyAsync(sig.data(), pp.qsig_all, 8ull * R * Qn, cudaMemcpyDeviceToHost, q->stream));
    SIGMO_CUDA_TRY(cudaMemcpyAsync(lab.data(), query->node_labels, Qn, cudaMemcpyDeviceToHost, q->stream));
  }
  SIGMO_CUDA_TRY(cudaStreamSynchronize(q->stream));

  // One pass over the signatures (vertex ranges in parallel): every vertex's
  // program as raw codes (its label, then (r << 8 | l << 4 | c) for each
  // non-zero counter in (r, l) order, rows of a fixed stride of 1 + 16 R
  // entries), marking the labels and thresholds that occur.  Plane ids are
  // assigned in label and (r, l, c) order, so raw codes sort like the plane
  // ids they map to.
  const uint32_t stride = 1 + 16 * R;
  std::vector<uint16_t> vraw(static_cast<size_t>(Qn) * stride);
  std::vector<uint32_t> vlen(Qn);
  const unsigned nt = host_threads(Qn);
  std::vector<std::vector<uint16_t>> thr_part(nt, std::vector<uint16_t>(static_cast<size_t>(R) * 16, 0));
  std::vector<std::vector<uint8_t>> lab_part(nt, std::vector<uint8_t>(256, 0));
  parallel_ranges(Qn, nt, [&](unsigned t, uint64_t v0, uint64_t v1) {
    uint16_t* tm = thr_part[t].data();
    uint8_t* lu = lab_part[t].data();
    for (uint64_t v = v0; v < v1; ++v) {
      uint16_t* row = vraw.data() + v * stride;
      uint32_t n = 0;
      lu[lab[v]] = 1;
      row[n++] = lab[v];
      for (uint32_t r = 0; r < R; ++r)
        for (uint64_t sv = sig[static_cast<size_t>(r) * Qn + v]; sv;) {
          const uint32_t l = static_cast<uint32_t>(__builtin_ctzll(sv)) >> 2, c = (sv >> (4 * l)) & 0xFu;
          tm[r * 16 + l] |= static_cast<uint16_t>(1u << c);
          row[n++] = static_cast<uint16_t>((r << 8) | (l << 4) | c);
          sv &= ~(0xFull << (4 * l));
        }
      vlen[v] = n;
    }
  });
  std::vector<uint8_t> label_used(256, 0);
  std::vector<uint16_t> thr_mask(static_cast<size_t>(R) * 16, 0);  // [r][l]: bit c = count c occurs
  for (unsigned t = 0; t < nt; ++t) {
    for (size_t i = 0; i < thr_mask.size(); ++i) thr_mask[i] |= thr_part[t][i];
    for (size_t i = 0; i < 256; ++i) label_used[i] |= lab_part[t][i];
  }
  // planes: label values used by queries (ascending), then the thresholds
  // (r, l, c) that occur, in (r, l, c) order
  std::vector<uint32_t> spec;
  std::vector<uint32_t> label_idx(256, 0), thr_idx(static_cast<size_t>(R) * 256, 0);
  for (uint32_t l = 0; l < 256; ++l)
    if (label_used[l]) {
      label_idx[l] = static_cast<uint32_t>(spec.size());
      spec.push_back(0x80000000u | l);
    }
  const uint32_t nlab = static_cast<uint32_t>(spec.size());
  for (uint32_t r = 0; r < R; ++r)
    for (uint32_t l = 0; l < 16; ++l)
      for (uint32_t c = 1; c < 16; ++c)
        if ((thr_mask[r * 16 + l] >> c) & 1u) {
          thr_idx[(r << 8) | (l << 4) | c] = static_cast<uint32_t>(spec.size());
          spec.push_back((r << 16) | (l << 8) | c);
        }
  if (spec.size() >= 65535) return fail(SIGMO_ERR_DOMAIN, "query batch needs %zu candidate planes (limit 65535)", spec.size());

  // classes: distinct (label, sig_1..sig_R), numbered in lexicographic program
  // order: the vertices sorted by (the first four raw codes packed high to low,
  // a shorter program's missing codes 0 so it sorts first; ties: the full
  // comparison), in parallel ranges merged pairwise
  struct Key {
    uint64_t k;
    uint32_t v;
  };
  std::vector<Key> keys(Qn);
  auto row_of = [&](uint32_t v) { return vraw.data() + static_cast<size_t>(v) * stride; };
  auto key_less = [&](const Key& x, const Key& y) {
    if (x.k != y.k) return x.k < y.k;
    return std::lexicographical_compare(row_of(x.v), row_of(x.v) + vlen[x.v], row_of(y.v), row_of(y.v) + vlen[y.v]);
  };
  std::vector<uint64_t> cut(nt + 1);
  for (unsigned t = 0; t <= nt; ++t) cut[t] = Qn * t / nt;
  parallel_ranges(Qn, nt, [&](unsigned, uint64_t v0, uint64_t v1) {
    for (uint64_t v = v0; v < v1; ++v) {
      const uint16_t* row = row_of(static_cast<uint32_t>(v));
      uint64_t k = 0;
      for (uint32_t i = 0; i < 4; ++i) k = (k << 16) | (i < vlen[v] ? row[i] : 0u);
      keys[v] = Key{k, static_cast<uint32_t>(v)};
    }
    std::sort(keys.begin() + v0, keys.begin() + v1, key_less);
  });
  for (unsigned w = 1; w < nt; w *= 2)  // pairwise merges of the sorted ranges
    parallel_ranges(nt, (nt + 2 * w - 1) / (2 * w), [&](unsigned, uint64_t g0, uint64_t g1) {
      for (uint64_t g = g0; g < g1; ++g) {
        const uint64_t a = 2 * w * g, m = std::min<uint64_t>(a + w, nt), b = std::min<uint64_t>(a + 2 * w, nt);
        if (m < b) std::inplace_merge(keys.begin() + cut[a], keys.begin() + cut[m], keys.begin() + cut[b], key_less);
      }
    }, 1);
  std::vector<uint32_t> cls(Qn), prog_off{0};
  std::vector<uint16_t> prog;
  prog.reserve(static_cast<size_t>(Qn) * 8);
  uint32_t max_len = 0;
  for (uint64_t i = 0; i < Qn; ++i) {
    const uint32_t v = keys[i].v;
    if (i == 0 || keys[i - 1].k != keys[i].k || vlen[keys[i - 1].v] != vlen[v] ||
        !std::equal(row_of(v), row_of(v) + vlen[v], row_of(keys[i - 1].v))) {
      const uint16_t* row = row_of(v);
      prog.push_back(static_cast<uint16_t>(label_idx[row[0]]));
      for (uint32_t j = 1; j < vlen[v]; ++j) prog.push_back(static_cast<uint16_t>(thr_idx[row[j]]));
      prog_off.push_back(static_cast<uint32_t>(prog.size()));
      max_len = std::max<uint32_t>(max_len, vlen[v]);
    }
    cls[v] = static_cast<uint32_t>(prog_off.size() - 2);
  }
  const uint32_t C = static_cast<uint32_t>(prog_off.size() - 1);
  std::vector<uint32_t> r_begin(R + 1, static_cast<uint32_t>(spec.size()));
  for (uint32_t k = nlab; k < spec.size(); ++k) {
    const uint32_t r = (spec[k] >> 16) & 0xFFu;
    r_begin[r] = std::min(r_begin[r], k);
  }
  for (int r = static_cast<int>(R) - 1; r >= 0; --r) r_begin[r] = std::min(r_begin[r], r_begin[r + 1]);
  pp.K = static_cast<uint32_t>(spec.size());
  pp.C = C;
  pp.nlab = nlab;
  SIGMO_TRY(upload(q, reinterpret_cast<void**>(&pp.spec), spec.data(), 4 * spec.size()));
  SIGMO_TRY(upload(q, reinterpret_cast<void**>(&pp.prog_off), prog_off.data(), 4 * prog_off.size()));
  SIGMO_TRY(upload(q, reinterpret_cast<void**>(&pp.prog), prog.data(), 2 * prog.size()));
  SIGMO_TRY(upload(q, reinterpret_cast<void**>(&pp.cls), cls.data(), 4 * cls.size()));
  SIGMO_TRY(upload(q, reinterpret_cast<void**>(&pp.r_begin), r_begin.data(), 4 * r_begin.size()));
  pp.h_spec = spec;
  pp.h_prog = prog;
  pp.h_prog_off = prog_off;
  pp.h_cls = cls;
  pp.h_qgoff = query->host_graph_offsets;
  pp.qc_for = nullptr;
  pp.max_len = max_len;
  SIGMO_CUDA_TRY(cudaStreamSynchronize(q->stream));  // host vectors go out of scope
  pp.R = R;
  pp.profile = q->opts.profile;
  pp.valid = true;
  return SIGMO_OK;
}

// Splits the query graphs into contiguous groups whose planes and classes fit
// one admission tile (kGroupSmemBudget), greedily in query order, and uploads
// each group's program in local plane / class ids.  off/list: every query
// graph's classes in evaluation order (global class ids).
int plan_groups(Queue* q, Graph* query, uint32_t AW, const std::vector<uint32_t>& off, const std::vector<uint32_t>& list) {
  PlaneProgram& pp = query->pp;
  const uint32_t QG = query->num_graphs, K = pp.K, C = pp.C, R = pp.R;
  std::vector<uint32_t> plane_mark(K, 0), class_mark(C, 0);  // stamp = group number + 1
  uint32_t stamp = 0, Kg = 0, q0 = 0;
  std::vector<std::pair<uint32_t, uint32_t>> ranges;
  auto query_adds = [&](uint32_t qg, uint32_t* dk) {  // planes query qg adds to the group
    *dk = 0;
    std::vector<uint32_t> seen_planes;
    for (uint32_t e = off[qg]; e < off[qg + 1]; ++e) {
      const uint32_t c = list[e];
      if (class_mark[c] == stamp) continue;
      for (uint32_t i = pp.h_prog_off[c]; i < pp.h_prog_off[c + 1]; ++i) {
        const uint32_t k = pp.h_prog[i];
        if (plane_mark[k] != stamp && std::find(seen_planes.begin(), seen_planes.end(), k) == seen_planes.end()) {
          seen_planes.push_back(k);
          ++*dk;
        }
      }
    }
  };
  auto take = [&](uint32_t qg) {
    for (uint32_t e = off[qg]; e < off[qg + 1]; ++e) {
      const uint32_t c = list[e];
      if (class_mark[c] == stamp) continue;
      class_mark[c] = stamp;
      for (uint32_t i = pp.h_prog_off[c]; i < pp.h_prog_off[c + 1]; ++i)
        if (plane_mark[pp.h_prog[i]] != stamp) {
          plane_mark[pp.h_prog[i]] = stamp;
          ++Kg;
        }
    }
  };
  stamp = 1;
  for (uint32_t qg = 0; qg < QG; ++qg) {
    uint32_t dk;
    query_adds(qg, &dk);
    if (qg > q0 && planes_admit_smem(Kg + dk, AW) > kGroupSmemBudget) {
      ranges.emplace_back(q0, qg);
      ++stamp;
      Kg = 0;
      q0 = qg;
    }
    take(qg);
    if (planes_admit_smem(Kg, AW) > 200u * 1024u)
      return fail(SIGMO_ERR_DOMAIN, "query graph %u alone needs more than one admission tile of shared memory", qg);
  }
  ranges.emplace_back(q0, QG);
  // each group's arrays, in local ids (planes in global order, so label
  // planes come first and thresholds stay grouped by iteration)
  for (size_t gi = 0; gi < ranges.size(); ++gi) {
    PlaneGroup grp;
    grp.q0 = ranges[gi].first;
    grp.q1 = ranges[gi].second;
    // this group's planes: those of its own queries' classes (marks from the
    // planning pass may have been overwritten by a later group sharing a plane)
    std::vector<uint8_t> in_group(K, 0);
    for (uint32_t qg = grp.q0; qg < grp.q1; ++qg)
      for (uint32_t e = off[qg]; e < off[qg + 1]; ++e)
        for (uint32_t i = pp.h_prog_off[list[e]]; i < pp.h_prog_off[list[e] + 1]; ++i) in_group[pp.h_prog[i]] = 1;
    std::vector<uint32_t> loc_plane(K, 0xFFFFFFFFu), spec, row_of, r_begin(R + 1, 0xFFFFFFFFu);
    for (uint32_t k = 0; k < K; ++k)
      if (in_group[k]) {
        loc_plane[k] = static_cast<uint32_t>(spec.size());
        spec.push_back(pp.h_spec[k]);
        row_of.push_back(k);
      }
    uint32_t nlab = 0;
    for (uint32_t i = 0; i < spec.size(); ++i) {
      if (spec[i] & 0x80000000u) {
        ++nlab;
      } else {
        const uint32_t r = (spec[i] >> 16) & 0xFFu;
        r_begin[r] = std::min(r_begin[r], i);
      }
    }
    r_begin[R] = static_cast<uint32_t>(spec.size());
    for (int r = static_cast<int>(R) - 1; r >= 0; --r) r_begin[r] = std::min(r_begin[r], r_begin[r + 1]);
    // local programs; qc: per query entry, its class's local program range
    std::vector<uint32_t> loc_class(C, 0xFFFFFFFFu), prog_off{0}, qc_off{0}, qc;
    std::vector<uint16_t> prog;
    for (uint32_t qg = grp.q0; qg < grp.q1; ++qg) {
      for (uint32_t e = off[qg]; e < off[qg + 1]; ++e) {
        const uint32_t c = list[e];
        if (loc_class[c] == 0xFFFFFFFFu) {
          loc_class[c] = static_cast<uint32_t>(prog_off.size() - 1);
          for (uint32_t i = pp.h_prog_off[c]; i < pp.h_prog_off[c + 1]; ++i)
            prog.push_back(static_cast<uint16_t>(loc_plane[pp.h_prog[i]]));
          prog_off.push_back(static_cast<uint32_t>(prog.size()));
        }
        qc.push_back(prog_off[loc_class[c]]);
        qc.push_back(prog_off[loc_class[c] + 1]);
      }
      qc_off.push_back(static_cast<uint32_t>(qc.size() / 2));
    }
    grp.K = static_cast<uint32_t>(spec.size());
    grp.C = static_cast<uint32_t>(prog_off.size() - 1);
    // every local id and range the kernel will index with must be inside its array
    for (uint16_t k : prog)
      if (k >= grp.K) return fail(SIGMO_ERR_INVALID, "internal: group %zu plane %u outside its %u planes", gi, k, grp.K);
    for (size_t i = 0; i < qc.size(); i += 2)
      if (qc[i] > qc[i + 1] || qc[i + 1] > prog.size())
        return fail(SIGMO_ERR_INVALID, "internal: group %zu program range outside its %zu entries", gi, prog.size());
    if (planes_admit_smem(grp.K, AW) > 200u * 1024u)
      return fail(SIGMO_ERR_DOMAIN, "group %zu needs more than one admission tile of shared memory", gi);
    grp.nlab = nlab;
    grp.n_qc = qc.size() / 2;
    grp.n_prog = prog.size();
    SIGMO_TRY(upload(q, reinterpret_cast<void**>(&grp.spec), spec.data(), 4 * spec.size()));
    SIGMO_TRY(upload(q, reinterpret_cast<void**>(&grp.r_begin), r_begin.data(), 4 * r_begin.size()));
    SIGMO_TRY(upload(q, reinterpret_cast<void**>(&grp.row_of), row_of.data(), 4 * row_of.size()));
    SIGMO_TRY(upload(q, reinterpret_cast<void**>(&grp.prog), prog.data(), 2 * prog.size()));
    SIGMO_TRY(upload(q, reinterpret_cast<void**>(&grp.qc_off), qc_off.data(), 4 * qc_off.size()));
    SIGMO_TRY(upload(q, reinterpret_cast<void**>(&grp.qc), qc.data(), 4 * qc.size()));
    SIGMO_CUDA_TRY(cudaStreamSynchronize(q->stream));  // host vectors go out of scope
    pp.groups.push_back(grp);
  }
  return SIGMO_OK;
}

// Per query graph, its distinct classes in the order the admission kernel
// evaluates them for `data`: rarest label first (the data graphs' vertex
// counts per label), then longer programs (more thresholds) first, so a
// query that a graph cannot admit is usually rejected by its first class.
int order_classes(Queue* q, Graph* query, Graph* data) {
  PlaneProgram& pp = query->pp;
  if (pp.qc && pp.qc_for == data && pp.qc_stamp == data->stamp) return SIGMO_OK;
  SIGMO_TRY(ensure_label_hist(q, data));
  const uint32_t QG = query->num_graphs;
  uint64_t all = 0;
  for (uint64_t x : data->label_hist) all += x;
  // query graphs in parallel ranges, each query's list on its own, then
  // concatenated in query order
  std::vector<std::vector<uint32_t>> per(QG);
  auto key = [&](uint32_t c) {
    const uint32_t lab = pp.h_spec[pp.h_prog[pp.h_prog_off[c]]] & 0xFFu;
    const uint64_t freq = lab == kWildcard ? all : data->label_hist[lab];
    return std::make_tuple(freq, 0u - (pp.h_prog_off[c + 1] - pp.h_prog_off[c]), c);
  };
  parallel_ranges(QG, host_threads(query->total_nodes), [&](unsigned, uint64_t q0, uint64_t q1) {
    for (uint64_t qg = q0; qg < q1; ++qg) {
      std::vector<uint32_t>& tmp = per[qg];
      // queries of one vertex are never admitted (gmcr.hpp:100): an empty list
      // tells the kernel so
      if (pp.h_qgoff[qg + 1] - pp.h_qgoff[qg] <= 1) continue;
      tmp.assign(pp.h_cls.begin() + pp.h_qgoff[qg], pp.h_cls.begin() + pp.h_qgoff[qg + 1]);
      std::sort(tmp.begin(), tmp.end());
      tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
      std::sort(tmp.begin(), tmp.end(), [&](uint32_t a, uint32_t b) { return key(a) < key(b); });
    }
  });
  std::vector<uint32_t> off{0}, list;
  for (uint32_t qg = 0; qg < QG; ++qg) {
    list.insert(list.end(), per[qg].begin(), per[qg].end());
    off.push_back(static_cast<uint32_t>(list.size()));
  }
  dev_free(q, pp.qc_off);
  dev_free(q, pp.qc);
  pp.qc_off = pp.qc = nullptr;
  // the kernel reads each entry as its class's program range [begin, end) in prog
  std::vector<uint32_t> ranges(2 * list.size());
  for (size_t e = 0; e < list.size(); ++e) {
    ranges[2 * e] = pp.h_prog_off[list[e]];
    ranges[2 * e + 1] = pp.h_prog_off[list[e] + 1];
  }
  SIGMO_TRY(upload(q, reinterpret_cast<void**>(&pp.qc_off), off.data(), 4 * off.size()));
  SIGMO_TRY(upload(q, reinterpret_cast<void**>(&pp.qc), ranges.data(), 4 * ranges.size()));
  pp.h_qc_n = list.size();
  free_groups(q, &pp);
  const uint32_t AW = data->adj_words;
  if (planes_admit_smem(pp.K, AW) > kGroupSmemBudget) SIGMO_TRY(plan_groups(q, query, AW, off, list));
  SIGMO_CUDA_TRY(cudaStreamSynchronize(q->stream));  // host vectors go out of scope
  pp.qc_for = data;
  pp.qc_stamp = data->stamp;
  return SIGMO_OK;
}

void release_plane_program(Graph* g) {
  if (g->pp.valid || g->pp.qsig_all) free_program(g->q, &g->pp);
}

}  // namespace sigmo_b200

using namespace sigmo_b200;

namespace {

struct Events {
  cudaEvent_t e[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  ~Events() {
    for (auto& x : e)
      if (x) cudaEventDestroy(x);
  }
};

// The literal join of graphs [0, L): one launch over every admitted query, or
// (serving) one per request's query range, so a request's counts do not
// depend on the other requests of its batch (the reference's work-items
// carry DFS state from one pair to the next, isomorphism.hpp:309).
int join_literal_ranges(Queue* q, Graph* query, Graph* data, const Candidates* c, Gmcr* m, int find_first, uint32_t L,
                        uint64_t* d_total, const BatchedRun& run) {
  if (!run.query_ranges || run.nranges == 0)
    return launch_join_literal(q, query, data, c, m, find_first, 0, L, d_total, 0, 0xFFFFFFFFu);
  for (uint32_t r = 0; r < run.nranges; ++r)
    SIGMO_TRY(launch_join_literal(q, query, data, c, m, find_first, 0, L, d_total, run.query_ranges[r], run.query_ranges[r + 1]));
  return SIGMO_OK;
}

// The bitset route: fused filter writes the final bitset (all words), GMCR
// and the join read it.  Used when the caller asks for the bitset, or when a
// batch does not fit the plane route.
int batched_bitset(Queue* q, Graph* query, Graph* data, uint32_t R, int find_first, Candidates* c, Gmcr* m,
                   uint64_t* d_total, Events& ev, const BatchedRun& run) {
  PlaneProgram& pp = query->pp;
  const uint64_t N = data->total_nodes;
  void* buf = nullptr;
  const uint64_t b_dsig = run.dsig ? 0 : 8ull * R * N, b_planes = 16ull * 16 * R * c->Wp;
  auto al = [](uint64_t x) { return (x + 255) & ~255ull; };
  SIGMO_TRY(tmp_alloc(q, &buf, al(b_dsig) + al(b_planes) + 256));
  uint64_t* dsig = run.dsig ? const_cast<uint64_t*>(run.dsig) : static_cast<uint64_t*>(buf);
  uint32_t* planes = reinterpret_cast<uint32_t*>(static_cast<char*>(buf) + al(b_dsig));
  int rc = run.dsig ? SIGMO_OK : launch_sig_all(q, data, R, dsig);
  for (uint32_t r = 0; r < R && !rc; ++r)
    rc = launch_sig_planes(q, dsig + static_cast<uint64_t>(r) * N, N, c->Wp, planes + static_cast<uint64_t>(r) * 16 * 4 * c->Wp);
  if (!rc && cudaEventRecord(ev.e[1], q->stream) != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "event record failed");
  if (!rc) rc = launch_fused_filter(q, query, data, R, pp.qsig_all, planes, c);
  if (!rc && cudaEventRecord(ev.e[2], q->stream) != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "event record failed");
  if (!rc) rc = launch_gmcr(q, query, data, c, m, true, 0);
  if (!rc && cudaEventRecord(ev.e[3], q->stream) != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "event record failed");
  const bool exact = q->opts.profile == kProfileExact;
  if (!rc && !exact) rc = join_literal_ranges(q, query, data, c, m, find_first, std::min(data->low_offset_graphs, data->num_graphs),
                                             d_total, run);
  if (!rc) rc = launch_join_fast(q, query, data, c, m, find_first, d_total);
  dev_free(q, buf);
  return rc;
}

// The plane route (no full bitset in HBM).
int batched_planes(Queue* q, Graph* query, Graph* data, uint32_t R, int find_first, Gmcr* m, uint64_t* d_total, Events& ev,
                   const BatchedRun& run) {
  // stage events are not recorded while the work is captured into a graph
  auto mark = [&](int i) -> int {
    if (run.capture) return SIGMO_OK;
    return cudaEventRecord(ev.e[i], q->stream) == cudaSuccess ? SIGMO_OK : fail(SIGMO_ERR_CUDA, "event record failed");
  };
  PlaneProgram& pp = query->pp;
  const uint64_t N = data->total_nodes, Qn = query->total_nodes;
  const uint32_t G = data->num_graphs, GW = (G + 31u) / 32u, AW = data->adj_words;
  const bool exact = q->opts.profile == kProfileExact;
  const uint32_t L = exact ? 0u : std::min(data->low_offset_graphs, G);
  // words of the bitset the literal join reads (graphs [0, L))
  const uint64_t Wlow = L ? (static_cast<uint64_t>(data->host_graph_offsets[L]) + 31) / 32 : 0;
  const uint64_t Wlp = (Wlow + 31) / 32 * 32;
  auto al = [](uint64_t x) { return (x + 255) & ~255ull; };
  const ResidentPlanes* rp = run.resident;
  const uint64_t b_dsig = run.dsig ? 0 : 8ull * R * N, b_planes = rp ? 0 : 8ull * GW * pp.K * AW * 32,
                 b_ne = 4ull * query->num_graphs * GW + 4ull * G;
  // resident planes: the batch's plane k is resident row row_map[k], and the
  // class programs are rewritten as resident rows for the join
  std::vector<uint32_t> row_map;
  std::vector<uint16_t> rprog;
  if (rp) {
    if (rp->R != R) return fail(SIGMO_ERR_INVALID, "resident planes hold %u iterations, the batch asks for %u", rp->R, R);
    row_map.resize(pp.K);
    for (uint32_t k = 0; k < pp.K; ++k) {
      const uint32_t sp = pp.h_spec[k];
      if (sp & 0x80000000u) {
        row_map[k] = rp->label_row[sp & 0xFFu];
      } else {
        const uint32_t r = (sp >> 16) & 0xFFu, l = (sp >> 8) & 0xFFu, c = sp & 0xFFu;
        row_map[k] = c <= rp->cmax[r * 16 + l] ? rp->base_row[r * 16 + l] + c - 1 : rp->zero_row;
      }
    }
    rprog.resize(pp.h_prog.size());
    for (size_t i = 0; i < rprog.size(); ++i) rprog[i] = static_cast<uint16_t>(row_map[pp.h_prog[i]]);
  }
  const uint64_t b_map = 4ull * row_map.size() + 2ull * rprog.size();
  const uint64_t b_lplanes = 16ull * 16 * R * Wlp, b_lbits = 4ull * Qn * Wlp;
  void* buf = nullptr;
  SIGMO_TRY(tmp_alloc(q, &buf, al(b_dsig) + al(b_planes) + al(b_ne) + al(b_lplanes) + al(b_lbits) + al(b_map) + 256));
  char* p = static_cast<char*>(buf);
  uint64_t* dsig = run.dsig ? const_cast<uint64_t*>(run.dsig) : reinterpret_cast<uint64_t*>(p);
  p += al(b_dsig);
  uint64_t* planes = reinterpret_cast<uint64_t*>(p);
  p += al(b_planes);
  uint32_t* admit = reinterpret_cast<uint32_t*>(p);  // [query graphs][GW], then per-graph counts [G]
  uint32_t* adm_counts = admit + static_cast<uint64_t>(query->num_graphs) * GW;
  p += al(b_ne);
  uint32_t* lplanes = reinterpret_cast<uint32_t*>(p);
  p += al(b_lplanes);
  uint32_t* lbits = reinterpret_cast<uint32_t*>(p);
  p += al(b_lbits);
  uint32_t* d_row_map = reinterpret_cast<uint32_t*>(p);
  uint16_t* d_rprog = reinterpret_cast<uint16_t*>(d_row_map + row_map.size());
  int rc = run.dsig ? SIGMO_OK : launch_sig_all(q, data, R, dsig);
  if (!rc && rp) {
    if (cudaMemcpyAsync(d_row_map, row_map.data(), 4ull * row_map.size(), cudaMemcpyHostToDevice, q->stream) != cudaSuccess ||
        cudaMemcpyAsync(d_rprog, rprog.data(), 2ull * rprog.size(), cudaMemcpyHostToDevice, q->stream) != cudaSuccess)
      rc = fail(SIGMO_ERR_CUDA, "H2D copy failed");
  }
  if (!rc) rc = mark(1);
  if (!rc) rc = order_classes(q, query, data);
  if (!rc && !rp && !pp.groups.empty()) {
    // a batch too large for one tile: group by group into the batch's planes
    if (cudaMemsetAsync(adm_counts, 0, 4ull * G, q->stream) != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "memset failed");
    for (size_t gi = 0; gi < pp.groups.size() && !rc; ++gi)
      rc = launch_planes_admit_group(q, query, data, dsig, R, pp.groups[gi], pp.K, planes, admit, adm_counts);
  } else if (!rc) {
    rc = rp ? launch_planes_admit_resident(q, query, data, *rp, pp, d_row_map, admit, adm_counts)
            : launch_planes_admit(q, query, data, dsig, R, pp, planes, admit, adm_counts);
  }
  if (!rc) rc = mark(2);
  // captured: the admitted total of the run that built the graph sizes the
  // arrays (the replay checks that it did not change)
  if (!rc) rc = launch_gmcr_from_admit(q, query, data, admit, adm_counts, m, !run.capture, run.capture ? m->total : 0);
  if (!rc) rc = mark(3);
  const bool literal = !rc && L && m->total;
  uint32_t reserve = 0;
  bool forked = false;  // the side stream joined this call's work
  if (literal) {
    // REF_PTX: graphs starting below vertex 256 keep the reference's live
    // `visited` bitset, so they take the literal join on the bitset words it
    // reads.  The words are computed here (a few KB per query vertex); the
    // literal join then runs on the side stream, overlapping the fast join,
    // which leaves one CTA slot per literal block free so that the literal
    // join does not wait behind its persistent CTAs.
    for (uint32_t r = 0; r < R && !rc; ++r)
      rc = launch_sig_planes(q, dsig + static_cast<uint64_t>(r) * N, N, Wlp, lplanes + static_cast<uint64_t>(r) * 16 * 4 * Wlp);
    if (!rc) rc = launch_fused_filter_raw(q, query->node_labels, pp.qsig_all, Qn, data->node_labels, N, lplanes, Wlp, R, lbits);
    const cudaStream_t main_stream = q->stream;
    if (!rc && (cudaEventRecord(q->ev_fork, main_stream) != cudaSuccess || cudaStreamWaitEvent(q->side, q->ev_fork, 0) != cudaSuccess))
      rc = fail(SIGMO_ERR_CUDA, "stream fork failed");
    forked = !rc;
    q->stream = q->side;
    reserve = std::min<uint32_t>(L, 148u);
    Candidates view;
    view.q = q;
    view.rows = Qn;
    view.targets = N;
    view.W = Wlow;
    view.Wp = Wlp;
    view.bits = lbits;
    if (!rc) rc = join_literal_ranges(q, query, data, &view, m, find_first, L, d_total, run);
    q->stream = main_stream;
  }
  if (!rc)
    rc = rp ? launch_join_fast_planes(q, query, data, pp, rp->planes, rp->rows, d_rprog, m, find_first, d_total, reserve)
            : launch_join_fast_planes(q, query, data, pp, planes, pp.K, pp.prog, m, find_first, d_total, reserve);
  // join the side stream back before the scratch is released and the total
  // read (only when this call forked it: a CUDA-graph capture may wait only
  // on events of streams that joined the capture)
  if (forked && (cudaEventRecord(q->ev_join, q->side) != cudaSuccess || cudaStreamWaitEvent(q->stream, q->ev_join, 0) != cudaSuccess))
    rc = rc ? rc : fail(SIGMO_ERR_CUDA, "stream join failed");
  dev_free(q, buf);
  return rc;
}

}  // namespace

namespace sigmo_b200 {

namespace {

void drop_graph(Gmcr* m) {
  if (m->graph) cudaGraphExecDestroy(m->graph);
  m->graph = nullptr;
  for (auto& k : m->graph_key) k = 0;
}

// Replays the captured batch: the device work of the planes route (no host
// synchronisation inside), then the match total and the GMCR total to the
// queue's pinned buffer.  Returns SIGMO_ERR_INVALID (and drops the graph)
// when the admitted total differs from the one the graph was sized for.
int replay_graph(Queue* q, Graph* query, Graph* data, Gmcr* m, sigmo_match_result* out) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  SIGMO_CUDA_TRY(cudaEventCreate(&e0));
  SIGMO_CUDA_TRY(cudaEventCreate(&e1));
  cudaError_t e = cudaEventRecord(e0, q->stream);
  if (e == cudaSuccess) e = cudaGraphLaunch(m->graph, q->stream);
  if (e == cudaSuccess) q->launches += m->graph_launches;
  if (e == cudaSuccess) e = cudaEventRecord(e1, q->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(q->stream);
  float f = 0;
  if (e == cudaSuccess) cudaEventElapsedTime(&f, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return fail(SIGMO_ERR_CUDA, "graph replay failed: %s", cudaGetErrorString(e));
  SIGMO_TRY(join_status_result(q));  // the graph read the status word back
  const uint64_t* pin = static_cast<const uint64_t*>(q->pinned);
  const uint32_t gtotal = *reinterpret_cast<const uint32_t*>(pin + 1);
  if (gtotal != m->total) {
    drop_graph(m);
    return fail(SIGMO_ERR_INVALID, "the admitted total changed since the graph was captured");
  }
  std::memset(out, 0, sizeof(*out));
  out->total_matches = pin[0];
  out->admitted_pairs = m->total;
  out->pairs = static_cast<uint64_t>(query->num_graphs) * data->num_graphs;
  out->ms_total = f;
  m->counts_valid = true;
  return SIGMO_OK;
}

// Captures the planes route for (query, data) into m->graph, sized by the
// admitted total of the run that just completed.
int capture_graph(Queue* q, Graph* query, Graph* data, uint32_t R, int find_first, Gmcr* m, const BatchedRun& run0) {
  drop_graph(m);
  BatchedRun run = run0;
  run.capture = true;
  Events ev;  // unused while capturing
  const uint64_t launches0 = q->launches;
  SIGMO_CUDA_TRY(cudaStreamBeginCapture(q->stream, cudaStreamCaptureModeThreadLocal));
  uint64_t* d_total = nullptr;
  int rc = join_status_reset(q);
  if (!rc) rc = tmp_alloc(q, reinterpret_cast<void**>(&d_total), 8);
  if (!rc && cudaMemsetAsync(d_total, 0, 8, q->stream) != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "memset failed");
  if (!rc) rc = batched_planes(q, query, data, R, find_first, m, d_total, ev, run);
  uint64_t* pin = static_cast<uint64_t*>(q->pinned);
  if (!rc && (cudaMemcpyAsync(pin, d_total, 8, cudaMemcpyDeviceToHost, q->stream) != cudaSuccess ||
              cudaMemcpyAsync(pin + 1, m->offsets + data->num_graphs, 4, cudaMemcpyDeviceToHost, q->stream) != cudaSuccess))
    rc = fail(SIGMO_ERR_CUDA, "capture of the read-back failed");
  if (!rc) rc = join_status_fetch(q);
  if (d_total) dev_free(q, d_total);
  cudaGraph_t g = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(q->stream, &g);
  if (!rc && ec != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "stream capture failed: %s", cudaGetErrorString(ec));
  if (!rc) {
    const cudaError_t ei = cudaGraphInstantiate(&m->graph, g, 0);
    if (ei != cudaSuccess) {
      m->graph = nullptr;
      rc = fail(SIGMO_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(ei));
    }
  }
  if (g) cudaGraphDestroy(g);
  cudaGetLastError();
  m->graph_launches = q->launches - launches0;
  q->launches = launches0;  // nothing ran during the capture
  m->counts_valid = true;   // the counts of the run before the capture are still in place
  return rc;
}

}  // namespace

int match_batched(Queue* q, Graph* query, Graph* data, uint32_t R, int find_first, bool materialize, Candidates* c, Gmcr* m,
                  sigmo_match_result* out, const BatchedRun& run, bool graph) {
  if (query->max_nodes > kMaxQueryNodes)
    return fail(SIGMO_ERR_DOMAIN, "query graphs of up to %u vertices are supported (largest: %u)", kMaxQueryNodes, query->max_nodes);
  if (data->max_nodes > 64u * kMaxAdjWords)
    return fail(SIGMO_ERR_DOMAIN, "the batched form supports data graphs of up to %u vertices (largest: %u)", 64u * kMaxAdjWords,
                data->max_nodes);
  if (q->opts.profile == kProfileX86)
    return fail(SIGMO_ERR_DOMAIN, "the batched form runs the REF_PTX and EXACT profiles; REF_X86 runs the stage-per-launch calls");
  SIGMO_CUDA_TRY(cudaSetDevice(q->device));
  const sigmo_tuning& tn = q->tune;
  const uint64_t key[7] = {query->stamp, data->stamp, R, static_cast<uint64_t>(find_first),
                           static_cast<uint64_t>(q->opts.profile) | (static_cast<uint64_t>(tn.overflow_serial) << 8) |
                               (static_cast<uint64_t>(tn.overflow_split) << 16) |
                               (static_cast<uint64_t>(tn.join_kernel) << 24) | (static_cast<uint64_t>(tn.join_pool) << 32),
                           (static_cast<uint64_t>(tn.join_blocks_per_sm) << 48) | (static_cast<uint64_t>(tn.join_chunk) << 40) |
                               (static_cast<uint64_t>(tn.mask_chunk_slots) << 32) | tn.overflow_blocks,
                           q->join_budget};
  if (graph && !materialize && m->graph && std::equal(key, key + 7, m->graph_key)) {
    const int rc = replay_graph(q, query, data, m, out);
    if (rc != SIGMO_ERR_INVALID) return rc;  // else: recapture below
  }
  drop_graph(m);  // this run may replace the arrays a captured batch refers to
  std::memset(out, 0, sizeof(*out));
  SIGMO_TRY(join_status_reset(q));
  Events ev;
  for (auto& e : ev.e) SIGMO_CUDA_TRY(cudaEventCreate(&e));
  SIGMO_CUDA_TRY(cudaEventRecord(ev.e[0], q->stream));
  // the data graph's signatures do not depend on the query batch: launched
  // first, they run while the host builds the query batch's plane program
  BatchedRun prun = run;
  uint64_t* dsig_tmp = nullptr;
  if (!run.dsig && !run.capture && R && data->total_nodes) {
    SIGMO_TRY(tmp_alloc(q, reinterpret_cast<void**>(&dsig_tmp), 8ull * R * data->total_nodes));
    const int src = launch_sig_all(q, data, R, dsig_tmp);
    if (src) {
      dev_free(q, dsig_tmp);
      return src;
    }
    prun.dsig = dsig_tmp;
  }
  struct FreeTmp {
    Queue* q;
    uint64_t* p;
    ~FreeTmp() { dev_free(q, p); }
  } free_dsig{q, dsig_tmp};
  SIGMO_TRY(build_plane_program(q, query, R));
  uint64_t* d_total = nullptr;
  SIGMO_TRY(tmp_alloc(q, reinterpret_cast<void**>(&d_total), 8));
  int rc = cudaMemsetAsync(d_total, 0, 8, q->stream) == cudaSuccess ? SIGMO_OK : fail(SIGMO_ERR_CUDA, "memset failed");
  // the planes route takes any batch whose query graphs each fit an admission
  // tile (larger batches are admitted in groups); planes take 8 B per
  // (plane, graph, word) in device memory
  int prc = order_classes(q, query, data);
  if (prc == SIGMO_ERR_DOMAIN) prc = SIGMO_OK;  // a query graph too large for a tile: bitset route
  else if (prc) return prc;
  const bool planes_fit = query->pp.qc_for == data && (!query->pp.groups.empty() ||
                                                       planes_admit_smem(query->pp.K, data->adj_words) <= 200u * 1024u);
  const bool bitset_route = materialize || !planes_fit;
  if (!rc && bitset_route && data->vertex_base)
    rc = fail(SIGMO_ERR_DOMAIN, "a shard (vertex base %u) runs on the planes route only; this batch needs the bitset route",
              data->vertex_base);
  if (!rc) {
    if (bitset_route) {
      sigmo_candidates_t cc = static_cast<sigmo_candidates_t>(c);
      if (!cc) rc = sigmo_candidates_create(static_cast<sigmo_queue_t>(q), query->total_nodes, data->total_nodes, &cc);
      if (!rc) rc = batched_bitset(q, query, data, R, find_first, cc, m, d_total, ev, prun);
      if (cc != c) sigmo_candidates_destroy(cc);
    } else {
      rc = batched_planes(q, query, data, R, find_first, m, d_total, ev, prun);
    }
  }
  if (!rc && cudaEventRecord(ev.e[4], q->stream) != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "event record failed");
  if (!rc) rc = join_status_fetch(q);
  if (!rc) {
    cudaError_t e = cudaMemcpyAsync(q->pinned, d_total, 8, cudaMemcpyDeviceToHost, q->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(q->stream);
    if (e != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "batched read-back failed: %s", cudaGetErrorString(e));
  }
  if (!rc) rc = join_status_result(q);
  if (!rc) {
    out->total_matches = *static_cast<uint64_t*>(q->pinned);
    out->admitted_pairs = m->total;
    out->pairs = static_cast<uint64_t>(query->num_graphs) * data->num_graphs;
    float f;
    cudaEventElapsedTime(&f, ev.e[0], ev.e[1]);
    out->ms_signatures = f;
    cudaEventElapsedTime(&f, ev.e[1], ev.e[2]);
    out->ms_filter = f;
    cudaEventElapsedTime(&f, ev.e[2], ev.e[3]);
    out->ms_mapping = f;
    cudaEventElapsedTime(&f, ev.e[3], ev.e[4]);
    out->ms_join = f;
    cudaEventElapsedTime(&f, ev.e[0], ev.e[4]);
    out->ms_total = f;
    m->counts_valid = true;
  }
  dev_free(q, d_total);
  if (!rc && graph && !bitset_route) {
    // graph mode: capture this batch for the next calls with the same inputs
    rc = capture_graph(q, query, data, R, find_first, m, run);
    if (!rc) std::copy(key, key + 7, m->graph_key);
  }
  return rc;
}

}  // namespace sigmo_b200

extern "C" int sigmo_match_batched(sigmo_queue_t q, sigmo_graph_t query, sigmo_graph_t data, uint32_t R, int find_first,
                                   uint32_t flags, sigmo_candidates_t c, sigmo_gmcr_t m, sigmo_match_result* out) {
  if (!q || !query || !data || !m || !out) return fail(SIGMO_ERR_INVALID, "null argument");
  const bool materialize = (flags & SIGMO_MATCH_MATERIALIZE_BITSET) != 0;
  if (materialize && !c) return fail(SIGMO_ERR_INVALID, "SIGMO_MATCH_MATERIALIZE_BITSET needs a candidates object");
  if (c && (c->rows != query->total_nodes || c->targets != data->total_nodes))
    return fail(SIGMO_ERR_INVALID, "candidate bitset does not match the graphs");
  if (m->q != q || (c && c->q != q) || query->q != q || data->q != q) return fail(SIGMO_ERR_INVALID, "handles belong to another queue");
  return match_batched(q, query, data, R, find_first, materialize, c, m, out, BatchedRun{},
                       (flags & SIGMO_MATCH_CUDA_GRAPH) != 0);
}

// ---- autotuner --------------------------------------------------------------
extern "C" int sigmo_autotune(sigmo_queue_t q, sigmo_graph_t query, sigmo_graph_t data, uint32_t R, int find_first,
                              uint32_t reps, sigmo_tuning* best, double* best_ms, double* default_ms) {
  if (!q || !query || !data || !best) return fail(SIGMO_ERR_INVALID, "null argument");
  if (query->q != q || data->q != q) return fail(SIGMO_ERR_INVALID, "handles belong to another queue");
  if (reps == 0) reps = 3;
  sigmo_gmcr_t m = nullptr;
  SIGMO_TRY(sigmo_gmcr_create(q, &m));
  const sigmo_tuning saved = q->tune;
  auto measure = [&](const sigmo_tuning& t, double* ms, uint64_t* total) -> int {
    q->tune = t;
    std::vector<double> js;
    sigmo_match_result r{};
    for (uint32_t i = 0; i <= reps; ++i) {
      SIGMO_TRY(match_batched(q, query, data, R, find_first, false, nullptr, m, &r, BatchedRun{}));
      if (i) js.push_back(r.ms_join);
    }
    std::sort(js.begin(), js.end());
    *ms = js[js.size() / 2];
    *total = r.total_matches;
    return SIGMO_OK;
  };
  sigmo_tuning cur = Queue{}.tune;  // the library default
  double cur_ms = 0, d_ms = 0;
  uint64_t d_total = 0, total = 0;
  int rc = measure(cur, &d_ms, &d_total);
  cur_ms = d_ms;
  struct Axis {
    uint32_t sigmo_tuning::*field;
    std::vector<uint32_t> values;
  };
  const Axis axes[] = {
      {&sigmo_tuning::join_kernel, {0, 1, 2}},
      {&sigmo_tuning::overflow_serial, {0, 1}},
      {&sigmo_tuning::join_blocks_per_sm, {1, 2, 3, 4}},
      {&sigmo_tuning::join_pool, {1, 2, 4, 8}},
      {&sigmo_tuning::join_chunk, {1, 2, 4, 8, 16}},
      {&sigmo_tuning::overflow_blocks, {148, 296, 592, 1184, 2368}},
      {&sigmo_tuning::mask_chunk_slots, {2, 8, 32}},
      {&sigmo_tuning::overflow_split, {1, 4, 16, 32}},
  };
  for (const Axis& ax : axes) {
    for (uint32_t v : ax.values) {
      if (rc) break;
      if (cur.*ax.field == v) continue;
      sigmo_tuning t = cur;
      t.*ax.field = v;
      double ms = 0;
      rc = measure(t, &ms, &total);
      if (!rc && total != d_total)
        rc = fail(SIGMO_ERR_INVALID, "autotune: a launch shape changed the result (%llu vs %llu)", (unsigned long long)total,
                  (unsigned long long)d_total);
      if (!rc && ms < cur_ms * 0.98) {
        cur = t;
        cur_ms = ms;
      }
    }
  }
  sigmo_gmcr_destroy(m);
  if (rc) {
    q->tune = saved;
    return rc;
  }
  q->tune = cur;
  *best = cur;
  if (best_ms) *best_ms = cur_ms;
  if (default_ms) *default_ms = d_ms;
  return SIGMO_OK;
}
