// Join kernels (isomorphism::join::joinCandidates, isomorphism.hpp:270-381).
//
// k_join_literal restates the reference's DFS step by step: one block per
// data graph, thread lid takes GMCR slots lid, lid+wg, ...; each pair runs the
// explicit-stack DFS in identity query order with the range-masked candidate
// count / k-th candidate (candidates.hpp:86-162), the uint8-indexed `visited`
// bitset (utils.hpp:64-96) and the induced adjacency check
// (isomorphism.hpp:150-168).  mapping[] starts zeroed per thread and is
// carried across the pairs the thread handles, as in the reference.  Under
// REF_PTX the visited bitset is inert for any data graph whose first vertex is
// >= 256; the batched form therefore runs this kernel only for the few graphs
// below that.
//
// k_join_fast counts the same matches with graph-local bit sets.  For the
// pairs it handles, the reference's count is order independent:
//   REF_PTX (visited inert): #{(d_0..d_{n-1}) in prod C_i : for all i<j,
//       adjQ(i,j) == adjD(d_i,d_j)}  (non-adjacent query vertices may share a
//       data vertex);
//   EXACT: the same with d injective.
// so each level's candidates are one AND over the earlier levels' adjacency
// rows, the last level is a popcount, and query vertices are placed in a
// connectivity order.  Find-first stops at the first match.
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.hpp"

namespace sigmo_b200 {
namespace {

// getCandidatesCount(src, s, e) on one bitset row.
__device__ __forceinline__ uint32_t cand_count(const uint32_t* __restrict__ row, uint32_t s, uint32_t e, int prof) {
  const uint32_t i0 = s >> 5, i1 = (e + 31u) >> 5;
  uint32_t c = 0;
  for (uint32_t i = i0; i < i1; ++i) c += __popc(row[i] & range_mask(i, s, e, prof));
  return c;
}

// getCandidateAt(src, idx, s, e): global id of the idx-th masked candidate.
__device__ __forceinline__ uint32_t cand_at(const uint32_t* __restrict__ row, uint32_t idx, uint32_t s, uint32_t e, int prof) {
  const uint32_t i0 = s >> 5, i1 = (e + 31u) >> 5;
  uint32_t c = 0;
  for (uint32_t i = i0; i < i1; ++i) {
    uint32_t blk = row[i] & range_mask(i, s, e, prof);
    const uint32_t bc = __popc(blk);
    if (c + bc > idx) {
      while (blk) {
        const uint32_t t = __ffs(blk) - 1;
        if (c == idx) return (i << 5) + t;
        blk &= blk - 1;
        ++c;
      }
    } else {
      c += bc;
    }
  }
  return 0xFFFFFFFFu;
}

// DeviceBatchedCSRGraph::isNeighbor (graph.hpp:72-77) for two vertices of
// data graph [s, e): via the local adjacency rows when the graph fits them.
__device__ __forceinline__ bool data_neighbor(uint32_t a, uint32_t b, uint32_t s, uint32_t ng, const uint64_t* __restrict__ adj,
                                              uint32_t AW, const uint32_t* __restrict__ roff, const uint32_t* __restrict__ col) {
  if (ng <= 64u * AW) {
    const uint32_t t = b - s;
    return (adj[static_cast<uint64_t>(a) * AW + (t >> 6)] >> (t & 63u)) & 1ull;
  }
  for (uint32_t i = roff[a]; i < roff[a + 1]; ++i)
    if (col[i] == b) return true;
  return false;
}

struct Frame {
  uint32_t depth;
  uint32_t idx;
};

template <bool EXACT>
__global__ void k_join_literal(const uint32_t* __restrict__ bits, uint64_t Wp, int prof,
                               const uint32_t* __restrict__ qgoff, const uint64_t* __restrict__ qadj,
                               const uint32_t* __restrict__ dgoff, const uint64_t* __restrict__ dadj, uint32_t dAW,
                               const uint32_t* __restrict__ droff, const uint32_t* __restrict__ dcol,
                               const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ indices, uint32_t g0,
                               uint32_t g1, int find_first, uint64_t* __restrict__ counts,
                               unsigned long long* __restrict__ d_total) {
  const uint32_t wg = blockDim.x, lid = threadIdx.x;
  uint64_t my_total = 0;
  for (uint32_t g = g0 + blockIdx.x; g < g1; g += gridDim.x) {
    const uint32_t s = dgoff[g], e = dgoff[g + 1], ng = e - s;
    const uint32_t seg0 = offsets[g], seglen = offsets[g + 1] - seg0;
    uint32_t mapping[kMaxQueryNodes + 1];
#pragma unroll 1
    for (uint32_t k = 0; k <= kMaxQueryNodes; ++k) mapping[k] = 0;
    for (uint32_t it = lid; it < seglen; it += wg) {
      const uint32_t qg = indices[seg0 + it];
      const uint32_t qoff = qgoff[qg], n = qgoff[qg + 1] - qoff;
      uint64_t found = 0;
      Frame stack[kMaxQueryNodes + 2];
      uint32_t top = 0;
      stack[top++] = {0u, 0u};
      if (!EXACT) {
        uint64_t visited = 0;  // Bitset<uint64_t>{offset = s}
        while (top > 0) {
          const Frame fr = stack[top - 1];
          const uint32_t qn = fr.depth;
          if (qn == n) {
            ++found;
            --top;
            if (find_first) break;
            continue;
          }
          const uint32_t* row = bits + static_cast<uint64_t>(qoff + qn) * Wp;
          if (fr.idx >= cand_count(row, s, e, prof)) {
            --top;
            visited &= ~refbit(mapping[qn], s);
            if (top == 1) visited = 0;
            continue;
          }
          const uint32_t cand = cand_at(row, fr.idx, s, e, prof);
          stack[top - 1].idx++;
          if (visited & refbit(cand, s)) continue;
          bool ok = true;
          for (uint32_t i = 0; i < qn && ok; ++i) {
            const bool qa = (qadj[qoff + i] >> qn) & 1ull;
            ok = qa == data_neighbor(mapping[i], cand, s, ng, dadj, dAW, droff, dcol);
          }
          if (ok) {
            mapping[qn] = cand;
            visited |= refbit(cand, s);
            stack[top++] = {qn + 1, 0u};
          }
        }
      } else {
        // Injective DFS with clean backtracking (graphs <= 256 vertices).
        uint64_t used[kMaxAdjWords] = {0, 0, 0, 0};
        uint32_t placed[kMaxQueryNodes + 1];
#pragma unroll 1
        for (uint32_t k = 0; k <= n; ++k) placed[k] = 0xFFFFFFFFu;
        while (top > 0) {
          const Frame fr = stack[top - 1];
          const uint32_t qn = fr.depth;
          if (qn == n) {
            ++found;
            --top;
            if (find_first) break;
            continue;
          }
          if (placed[qn] != 0xFFFFFFFFu) {
            const uint32_t t = placed[qn] - s;
            used[t >> 6] &= ~(1ull << (t & 63u));
            placed[qn] = 0xFFFFFFFFu;
          }
          const uint32_t* row = bits + static_cast<uint64_t>(qoff + qn) * Wp;
          if (fr.idx >= cand_count(row, s, e, prof)) {
            --top;
            continue;
          }
          const uint32_t cand = cand_at(row, fr.idx, s, e, prof);
          stack[top - 1].idx++;
          const uint32_t t = cand - s;
          if ((used[t >> 6] >> (t & 63u)) & 1ull) continue;
          bool ok = true;
          for (uint32_t i = 0; i < qn && ok; ++i) {
            const bool qa = (qadj[qoff + i] >> qn) & 1ull;
            ok = qa == data_neighbor(mapping[i], cand, s, ng, dadj, dAW, droff, dcol);
          }
          if (ok) {
            mapping[qn] = cand;
            placed[qn] = cand;
            used[t >> 6] |= 1ull << (t & 63u);
            stack[top++] = {qn + 1, 0u};
          }
        }
      }
      counts[seg0 + it] = found;
      my_total += found;
    }
  }
  // block reduction, one atomic per block
  for (int o = 16; o; o >>= 1) my_total += __shfl_xor_sync(0xFFFFFFFFu, my_total, o);
  __shared__ uint64_t part[32];
  if ((lid & 31u) == 0) part[lid >> 5] = my_total;
  __syncthreads();
  if (lid < 32) {
    uint64_t v = lid < ((wg + 31u) >> 5) ? part[lid] : 0ull;
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if (lid == 0 && v) atomicAdd(d_total, static_cast<unsigned long long>(v));
  }
}

// Graph-local candidate set of one bitset row for data graph [s, e): bit t =
// global candidate s + t, after the profile's range masks.
template <int AW>
__device__ __forceinline__ void extract_local(const uint32_t* __restrict__ row, uint32_t s, uint32_t e, int prof, uint64_t* out) {
#pragma unroll
  for (int k = 0; k < AW; ++k) out[k] = 0;
  const uint32_t i0 = s >> 5, i1 = (e + 31u) >> 5;
  for (uint32_t i = i0; i < i1; ++i) {
    uint32_t wv = row[i] & range_mask(i, s, e, prof);
    if (!wv) continue;
    int32_t off = static_cast<int32_t>(i << 5) - static_cast<int32_t>(s);
    if (off < 0) {
      wv >>= static_cast<uint32_t>(-off);
      off = 0;
    }
    const uint32_t k = static_cast<uint32_t>(off) >> 6, sh = static_cast<uint32_t>(off) & 63u;
#pragma unroll
    for (int kk = 0; kk < AW; ++kk) {
      if (static_cast<uint32_t>(kk) == k) out[kk] |= static_cast<uint64_t>(wv) << sh;
      if (sh > 32u && static_cast<uint32_t>(kk) == k + 1) out[kk] |= static_cast<uint64_t>(wv) >> (64u - sh);
    }
  }
}

// Candidate set of query vertex v (global id) in data graph g from the plane
// tiles: the AND of the planes of v's class program.
template <int AW>
__device__ __forceinline__ void mask_from_planes(const uint64_t* __restrict__ planes, uint32_t K, uint32_t g, uint32_t cls_v,
                                                 const uint32_t* __restrict__ prog_off, const uint16_t* __restrict__ prog,
                                                 uint64_t* out) {
  const uint64_t* base = planes + static_cast<uint64_t>(g >> 5) * K * AW * 32 + (g & 31u);
#pragma unroll
  for (int w = 0; w < AW; ++w) out[w] = ~0ull;
  const uint32_t e1 = prog_off[cls_v + 1];
  for (uint32_t e = prog_off[cls_v]; e < e1; ++e) {
    const uint32_t k = prog[e];
#pragma unroll
    for (int w = 0; w < AW; ++w) out[w] &= base[(static_cast<uint64_t>(k) * AW + w) * 32];
  }
}

template <int AW, bool EXACT, bool FROM_PLANES>
__global__ void __launch_bounds__(128) k_join_fast(
    const uint32_t* __restrict__ bits, uint64_t Wp, const uint64_t* __restrict__ planes, uint32_t K,
    const uint32_t* __restrict__ prog_off, const uint16_t* __restrict__ prog, const uint32_t* __restrict__ cls,
    int prof, const uint32_t* __restrict__ qgoff,
    const uint8_t* __restrict__ qorder, const uint64_t* __restrict__ qsel, const uint64_t* __restrict__ qsel_id,
    const uint8_t* __restrict__ qsym, const uint32_t* __restrict__ dgoff, const uint64_t* __restrict__ dadj,
    const uint8_t* __restrict__ dsym, const uint32_t* __restrict__ indices, const uint32_t* __restrict__ pair_graph,
    uint64_t total, uint32_t skip_below, int find_first, unsigned long long* __restrict__ cursor,
    uint64_t* __restrict__ counts, unsigned long long* __restrict__ d_total) {
  constexpr uint32_t kChunk = 8;  // slots per lane per warp grab
  const unsigned lane = threadIdx.x & 31u;
  uint64_t my_total = 0;
  uint64_t M[kMaxQueryNodes][AW];     // candidates of each level (graph-local)
  uint64_t cand[kMaxQueryNodes][AW];  // untried candidates of each level
  uint64_t rows[kMaxQueryNodes][AW];  // adjacency row of each level's pick
  uint32_t pick[kMaxQueryNodes];
  for (;;) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(cursor, 32ull * kChunk);
    base = __shfl_sync(0xFFFFFFFFu, base, 0);
    if (base >= total) break;
    for (uint32_t c = 0; c < kChunk; ++c) {
      const uint64_t slot = base + c * 32ull + lane;
      if (slot >= total) break;
      const uint32_t g = pair_graph[slot];
      if (g < skip_below) continue;
      const uint32_t qg = indices[slot];
      const uint32_t qoff = qgoff[qg], n = qgoff[qg + 1] - qoff;
      const uint32_t s = dgoff[g], e = dgoff[g + 1];
      const bool ident = !(qsym[qg] && dsym[g]);
      const uint64_t* selp = (ident ? qsel_id : qsel) + qoff;
      for (uint32_t k = 0; k < n; ++k) {
        const uint32_t v = ident ? k : qorder[qoff + k];
        if (FROM_PLANES) mask_from_planes<AW>(planes, K, g, cls[qoff + v], prog_off, prog, M[k]);
        else extract_local<AW>(bits + static_cast<uint64_t>(qoff + v) * Wp, s, e, prof, M[k]);
      }
#pragma unroll
      for (int w = 0; w < AW; ++w) cand[0][w] = M[0][w];
      uint64_t cnt = 0;
      int k = 0;
      while (k >= 0) {
        bool empty = true;
#pragma unroll
        for (int w = 0; w < AW; ++w) empty &= cand[k][w] == 0;
        if (empty) {
          --k;
          continue;
        }
        uint32_t t = 0;
#pragma unroll
        for (int w = AW - 1; w >= 0; --w)
          if (cand[k][w]) t = 64u * w + (__ffsll(static_cast<long long>(cand[k][w])) - 1);
        cand[k][t >> 6] &= cand[k][t >> 6] - 1;
        pick[k] = t;
        const uint64_t* r = dadj + static_cast<uint64_t>(s + t) * AW;
#pragma unroll
        for (int w = 0; w < AW; ++w) rows[k][w] = r[w];
        const uint64_t sl = selp[k + 1];
        uint64_t nx[AW], excl[AW];
#pragma unroll
        for (int w = 0; w < AW; ++w) {
          nx[w] = M[k + 1][w];
          excl[w] = 0;
        }
        for (int i = 0; i <= k; ++i) {
          const bool adjq = (sl >> i) & 1ull;
#pragma unroll
          for (int w = 0; w < AW; ++w) nx[w] &= adjq ? rows[i][w] : ~rows[i][w];
          if (EXACT) {
#pragma unroll
            for (int w = 0; w < AW; ++w)
              if ((pick[i] >> 6) == static_cast<uint32_t>(w)) excl[w] |= 1ull << (pick[i] & 63u);
          }
        }
        if (EXACT) {
#pragma unroll
          for (int w = 0; w < AW; ++w) nx[w] &= ~excl[w];
        }
        if (static_cast<uint32_t>(k + 1) == n - 1) {
          uint32_t pc = 0;
#pragma unroll
          for (int w = 0; w < AW; ++w) pc += __popcll(nx[w]);
          cnt += pc;
          if (find_first && cnt) break;
          continue;
        }
        ++k;
#pragma unroll
        for (int w = 0; w < AW; ++w) cand[k][w] = nx[w];
      }
      if (find_first && cnt) cnt = 1;
      counts[slot] = cnt;
      my_total += cnt;
    }
  }
  for (int o = 16; o; o >>= 1) my_total += __shfl_xor_sync(0xFFFFFFFFu, my_total, o);
  if (lane == 0 && my_total) atomicAdd(d_total, static_cast<unsigned long long>(my_total));
}

}  // namespace

int launch_join_literal(Queue* q, const Graph* query, const Graph* data, const Candidates* c, Gmcr* m, int find_first,
                        uint32_t graph_begin, uint32_t graph_end, uint64_t* d_total) {
  if (graph_end <= graph_begin) return SIGMO_OK;
  if (query->max_nodes > kMaxQueryNodes)
    return fail(SIGMO_ERR_DOMAIN, "query graphs of up to %u vertices are supported (largest: %u)", kMaxQueryNodes, query->max_nodes);
  const bool exact = q->opts.profile == kProfileExact;
  if (exact && data->max_nodes > 64u * kMaxAdjWords)
    return fail(SIGMO_ERR_DOMAIN, "exact profile supports data graphs of at most %u vertices", 64u * kMaxAdjWords);
  const uint32_t wg = q->opts.join_work_group_size ? q->opts.join_work_group_size : 128u;
  if (wg > 1024u || (wg & 31u)) return fail(SIGMO_ERR_INVALID, "join work-group size %u must be a multiple of 32 <= 1024", wg);
  const unsigned grid = std::min<uint32_t>(graph_end - graph_begin, 148u * 64u);
  auto* tot = reinterpret_cast<unsigned long long*>(d_total);
  if (exact)
    k_join_literal<true><<<grid, wg, 0, q->stream>>>(c->bits, c->Wp, q->opts.profile, query->graph_offsets, query->adj,
                                                      data->graph_offsets, data->adj, data->adj_words, data->row_offsets,
                                                      data->column_indices, m->offsets, m->indices, graph_begin, graph_end,
                                                      find_first, m->counts, tot);
  else
    k_join_literal<false><<<grid, wg, 0, q->stream>>>(c->bits, c->Wp, q->opts.profile, query->graph_offsets, query->adj,
                                                       data->graph_offsets, data->adj, data->adj_words, data->row_offsets,
                                                       data->column_indices, m->offsets, m->indices, graph_begin, graph_end,
                                                       find_first, m->counts, tot);
  return check_launch(q, "k_join_literal");
}

int launch_join_fast(Queue* q, const Graph* query, const Graph* data, const Candidates* c, Gmcr* m, int find_first,
                     uint64_t* d_total) {
  if (!m->total) return SIGMO_OK;
  if (query->max_nodes > kMaxQueryNodes)
    return fail(SIGMO_ERR_DOMAIN, "query graphs of up to %u vertices are supported (largest: %u)", kMaxQueryNodes, query->max_nodes);
  const bool exact = q->opts.profile == kProfileExact;
  if (data->max_nodes > 64u * kMaxAdjWords)
    return fail(SIGMO_ERR_DOMAIN, "the batched join supports data graphs of at most %u vertices", 64u * kMaxAdjWords);
  SIGMO_TRY(launch_query_order(const_cast<Graph*>(query)));
  void* scratch = nullptr;
  SIGMO_TRY(queue_scratch(q, 256, &scratch));
  auto* cursor = static_cast<unsigned long long*>(scratch);
  SIGMO_CUDA_TRY(cudaMemsetAsync(cursor, 0, sizeof(unsigned long long), q->stream));
  const uint32_t skip = exact ? 0u : data->low_offset_graphs;
  const unsigned block = 128;
  const unsigned grid = grid_for((m->total + 31) / 32 * 32, block, 148u * 16u);
  auto* tot = reinterpret_cast<unsigned long long*>(d_total);
#define SIGMO_JOIN_FAST(AWV, EX)                                                                                    \
  k_join_fast<AWV, EX, false><<<grid, block, 0, q->stream>>>(c->bits, c->Wp, nullptr, 0, nullptr, nullptr, nullptr,         \
                                                       q->opts.profile, query->graph_offsets, query->qorder,             \
                                                       query->qsel, query->qsel_id, query->sym, data->graph_offsets,     \
                                                       data->adj, data->sym, m->indices, m->pair_graph, m->total, skip,  \
                                                       find_first, cursor, m->counts, tot)
  switch (data->adj_words) {
    case 1: if (exact) SIGMO_JOIN_FAST(1, true); else SIGMO_JOIN_FAST(1, false); break;
    case 2: if (exact) SIGMO_JOIN_FAST(2, true); else SIGMO_JOIN_FAST(2, false); break;
    default: if (exact) SIGMO_JOIN_FAST(4, true); else SIGMO_JOIN_FAST(4, false); break;
  }
#undef SIGMO_JOIN_FAST
  return check_launch(q, "k_join_fast");
}

int launch_join_fast_planes(Queue* q, const Graph* query, const Graph* data, const PlaneProgram& pp, const uint64_t* planes,
                            Gmcr* m, int find_first, uint64_t* d_total) {
  if (!m->total) return SIGMO_OK;
  if (query->max_nodes > kMaxQueryNodes)
    return fail(SIGMO_ERR_DOMAIN, "query graphs of up to %u vertices are supported (largest: %u)", kMaxQueryNodes, query->max_nodes);
  const bool exact = q->opts.profile == kProfileExact;
  SIGMO_TRY(launch_query_order(const_cast<Graph*>(query)));
  void* cur = nullptr;
  SIGMO_TRY(dev_alloc(q, &cur, 256));
  auto* cursor = static_cast<unsigned long long*>(cur);
  SIGMO_CUDA_TRY(cudaMemsetAsync(cursor, 0, sizeof(unsigned long long), q->stream));
  const uint32_t skip = exact ? 0u : data->low_offset_graphs;
  const unsigned block = 128;
  const unsigned grid = grid_for((m->total + 31) / 32 * 32, block, 148u * 16u);
  auto* tot = reinterpret_cast<unsigned long long*>(d_total);
#define SIGMO_JOIN_PLANES(AWV, EX)                                                                                      \
  k_join_fast<AWV, EX, true><<<grid, block, 0, q->stream>>>(nullptr, 0, planes, pp.K, pp.prog_off, pp.prog, pp.cls,      \
                                                            q->opts.profile, query->graph_offsets, query->qorder,        \
                                                            query->qsel, query->qsel_id, query->sym, data->graph_offsets, \
                                                            data->adj, data->sym, m->indices, m->pair_graph, m->total,   \
                                                            skip, find_first, cursor, m->counts, tot)
  switch (data->adj_words) {
    case 1: if (exact) SIGMO_JOIN_PLANES(1, true); else SIGMO_JOIN_PLANES(1, false); break;
    case 2: if (exact) SIGMO_JOIN_PLANES(2, true); else SIGMO_JOIN_PLANES(2, false); break;
    default: if (exact) SIGMO_JOIN_PLANES(4, true); else SIGMO_JOIN_PLANES(4, false); break;
  }
#undef SIGMO_JOIN_PLANES
  int rc = check_launch(q, "k_join_fast<planes>");
  dev_free(q, cur);
  return rc;
}

}  // namespace sigmo_b200
