// Graph-derived device structures and the signature kernels.
//
// Signatures follow Signature<PowerGraph,4> (library/include/signature.hpp):
// generateCSRSignatures (:125-152) and refineCSRSignatures<PowerGraph>
// (:336-390).  The refinement is a bounded BFS per vertex; here each graph's
// local adjacency is kept as one bit row per vertex (u64 words, local ids), so
// a BFS level is an OR of rows selected by the frontier's bits.
#include <cuda_runtime.h>

#include "bulk.cuh"
#include "internal.hpp"

namespace sigmo_b200 {
namespace {

__global__ void k_node_graph(const uint32_t* __restrict__ goff, uint32_t G, uint32_t* __restrict__ node_graph) {
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < G; g += gridDim.x * blockDim.x) {
    const uint32_t v1 = goff[g + 1];
    for (uint32_t v = goff[g]; v < v1; ++v) node_graph[v] = g;
  }
}

// Local adjacency rows: bit t of row v = (prev + t) appears in v's CSR row,
// for local ids t < 64 * AW (prev = first vertex of v's graph).
template <int AW>
__global__ void k_build_adj(uint64_t N, const uint32_t* __restrict__ roff, const uint32_t* __restrict__ col,
                            const uint32_t* __restrict__ goff, const uint32_t* __restrict__ node_graph,
                            uint64_t* __restrict__ adj) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < N; v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t g = node_graph[v];
    const uint32_t prev = goff[g], n = goff[g + 1] - prev;
    uint64_t row[AW];
#pragma unroll
    for (int k = 0; k < AW; ++k) row[k] = 0;
    for (uint32_t i = roff[v]; i < roff[v + 1]; ++i) {
      const uint32_t t = col[i] - prev;  // neighbours outside the graph set no bit
      if (t < n && t < 64u * AW) {
#pragma unroll
        for (int k = 0; k < AW; ++k)
          if ((t >> 6) == (uint32_t)k) row[k] |= 1ull << (t & 63u);
      }
    }
#pragma unroll
    for (int k = 0; k < AW; ++k) adj[v * AW + k] = row[k];
  }
}

// generateCSRSignatures (signature.hpp:136-146): +1 per neighbour label, on
// top of the current value.
__global__ void k_sig_generate(uint64_t N, const uint32_t* __restrict__ roff, const uint32_t* __restrict__ col,
                               const uint8_t* __restrict__ lab, uint64_t* __restrict__ sig) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < N; v += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t s = sig[v];
    for (uint32_t i = roff[v]; i < roff[v + 1]; ++i) s = sig_inc(s, lab[col[i]]);
    sig[v] = s;
  }
}

// REF_PTX BFS for graphs of more than 256 vertices: the reference's bitset
// truncates local ids to uint8_t, so vertex t occupies bit (t & 255) when that
// is < 64 and no bit otherwise; bit b is expanded through vertex prev + b.
__device__ uint64_t ptx_wide_ball(uint32_t v, uint32_t prev, uint32_t view, const uint32_t* __restrict__ roff,
                                  const uint32_t* __restrict__ col, uint64_t* self_bit) {
  const uint64_t self = refbit(v - prev, 0);
  uint64_t F = self, R = self;
  for (uint32_t it = 0; it < view && F; ++it) {
    uint64_t nx = 0, m = F;
    while (m) {
      const uint32_t b = __ffsll(static_cast<long long>(m)) - 1;
      m &= m - 1;
      const uint32_t u = prev + b;
      for (uint32_t i = roff[u]; i < roff[u + 1]; ++i) nx |= refbit(col[i] - prev, 0);
    }
    nx &= ~R;
    R |= nx;
    F = nx;
  }
  *self_bit = self;
  return R;
}

// refineCSRSignatures<PowerGraph> (signature.hpp:348-386), REF_PTX profile:
// sphere = ball_view(v) \ {v} \ old(v); sig = label histogram of the sphere;
// old |= sphere.  Local ids >= 64 have no bit (graph sizes <= 256).
// X86 (REF_X86, graphs of <= 256 vertices): the 64-bit sets take local id
// mod 64 (Bitset<uint64_t> with the shift count modulo 64), so a vertex's
// neighbours land on their ids mod 64 (its adjacency words ORed together),
// and the frontier's bit b expands vertex b of the graph.
template <bool X86>
__global__ void k_sig_refine_ptx(uint64_t N, const uint32_t* __restrict__ goff, const uint32_t* __restrict__ node_graph,
                                 const uint64_t* __restrict__ adj, uint32_t AW, const uint32_t* __restrict__ roff,
                                 const uint32_t* __restrict__ col, const uint8_t* __restrict__ lab, uint32_t view,
                                 uint64_t* __restrict__ sig, uint64_t* __restrict__ reach) {
  for (uint64_t vv = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; vv < N; vv += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = static_cast<uint32_t>(vv);
    const uint32_t g = node_graph[v];
    const uint32_t prev = goff[g], n = goff[g + 1] - prev;
    uint64_t self, R;
    if (!X86 && n > 256u) {
      R = ptx_wide_ball(v, prev, view, roff, col, &self);
    } else {
      const uint32_t lv = v - prev;
      self = X86 ? (1ull << (lv & 63u)) : (lv < 64u ? (1ull << lv) : 0ull);
      uint64_t F = self;
      R = self;
      for (uint32_t it = 0; it < view && F; ++it) {
        uint64_t nx = 0, m = F;
        while (m) {
          const uint32_t b = __ffsll(static_cast<long long>(m)) - 1;
          m &= m - 1;
          const uint64_t* row = adj + static_cast<uint64_t>(prev + b) * AW;
          if (X86) {
            for (uint32_t k = 0; k < AW; ++k) nx |= row[k];
          } else {
            nx |= row[0];
          }
        }
        nx &= ~R;
        R |= nx;
        F = nx;
      }
    }
    R &= ~self;
    const uint64_t old = reach[v];
    uint64_t sphere = R & ~old;
    const uint64_t keep = sphere;
    uint64_t s = 0;
    while (sphere) {
      const uint32_t b = __ffsll(static_cast<long long>(sphere)) - 1;
      sphere &= sphere - 1;
      s = sig_inc(s, lab[prev + b]);
    }
    sig[v] = s;
    reach[v] = keep | old;
  }
}

// EXACT profile: true local sets of up to 64*AW vertices.
template <int AW>
__global__ void k_sig_refine_exact(uint64_t N, const uint32_t* __restrict__ goff, const uint32_t* __restrict__ node_graph,
                                   const uint64_t* __restrict__ adj, const uint8_t* __restrict__ lab, uint32_t view,
                                   uint64_t* __restrict__ sig, uint64_t* __restrict__ reach) {
  for (uint64_t vv = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; vv < N; vv += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = static_cast<uint32_t>(vv);
    const uint32_t prev = goff[node_graph[v]];
    const uint32_t lv = v - prev;
    uint64_t F[AW], R[AW];
#pragma unroll
    for (int k = 0; k < AW; ++k) F[k] = R[k] = ((lv >> 6) == (uint32_t)k) ? (1ull << (lv & 63u)) : 0ull;
    for (uint32_t it = 0; it < view; ++it) {
      bool any = false;
#pragma unroll
      for (int k = 0; k < AW; ++k) any |= F[k] != 0;
      if (!any) break;
      uint64_t nx[AW];
#pragma unroll
      for (int k = 0; k < AW; ++k) nx[k] = 0;
#pragma unroll
      for (int w = 0; w < AW; ++w) {
        uint64_t m = F[w];
        while (m) {
          const uint32_t b = __ffsll(static_cast<long long>(m)) - 1 + 64u * w;
          m &= m - 1;
          const uint64_t* row = adj + static_cast<uint64_t>(prev + b) * AW;
#pragma unroll
          for (int k = 0; k < AW; ++k) nx[k] |= row[k];
        }
      }
#pragma unroll
      for (int k = 0; k < AW; ++k) {
        nx[k] &= ~R[k];
        R[k] |= nx[k];
        F[k] = nx[k];
      }
    }
    uint64_t s = 0;
#pragma unroll
    for (int k = 0; k < AW; ++k) {
      if ((lv >> 6) == (uint32_t)k) R[k] &= ~(1ull << (lv & 63u));
      uint64_t* old = reach + static_cast<uint64_t>(v) * kMaxAdjWords + k;
      uint64_t sphere = R[k] & ~*old;
      *old |= R[k];
      while (sphere) {
        const uint32_t b = __ffsll(static_cast<long long>(sphere)) - 1;
        sphere &= sphere - 1;
        s = sig_inc(s, lab[prev + 64u * k + b]);
      }
    }
    sig[v] = s;
  }
}

// All refinement iterations 1..R at once (batched form): starting from empty
// reachables, iteration r's sphere is exactly BFS level r, so one BFS to
// depth R emits every iteration's signature.  sig_all is [R][N].
//
// Each CTA's graphs are staged on chip.  A CTA takes 256 consecutive
// vertices; they belong to a run of whole graphs whose adjacency rows
// [row_lo, row_hi) (at most 256 + 128 * AW rows for graphs of up to 64 * AW
// vertices) arrive in shared memory by one bulk asynchronous copy (the TMA
// engine, cp.async.bulk, completion counted on an mbarrier), and whose labels
// arrive by plain loads meanwhile; every vertex's BFS then reads shared memory
// only.  The copy starts on a 16-byte boundary of the adjacency array, is a
// multiple of 16 bytes and ends inside the array (a last 8-byte row past the
// final 16-byte boundary is loaded by a thread).  A range whose graphs do not
// fit (wide graphs) reads global memory instead.  The mbarrier
// wait is bounded; past the bound the range is computed from global memory
// (results are the same either way) and the CTA stops staging.
constexpr uint32_t kSigRange = 256;
template <int AW, bool EXACT>
__global__ void __launch_bounds__(kSigRange) k_sig_all_staged(uint64_t N, const uint32_t* __restrict__ goff,
                                                              const uint32_t* __restrict__ node_graph,
                                                              const uint64_t* __restrict__ adj,
                                                              const uint32_t* __restrict__ roff,
                                                              const uint32_t* __restrict__ col,
                                                              const uint8_t* __restrict__ lab, uint32_t Rn,
                                                              uint64_t* __restrict__ sig_all) {
  constexpr uint32_t kCap = kSigRange + 128u * AW;         // rows of one range's graphs, at most
  __shared__ __align__(16) uint64_t s_rows[kCap * AW + 2];  // + 16 bytes: the copy may start one row early
  __shared__ uint8_t s_lab[kCap];
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ int s_ok;  // the CTA still stages (no wait has run out)
  const uint64_t adj_bytes = N * AW * 8ull;
  if (threadIdx.x == 0) {
    mbar_init(&s_bar, 1);
    s_ok = 1;
  }
  __syncthreads();
  uint32_t parity = 0;
  for (uint64_t v0 = static_cast<uint64_t>(blockIdx.x) * kSigRange; v0 < N; v0 += static_cast<uint64_t>(gridDim.x) * kSigRange) {
    const uint64_t v1 = v0 + kSigRange < N ? v0 + kSigRange : N;
    const uint32_t row_lo = goff[node_graph[v0]], row_hi = goff[node_graph[v1 - 1] + 1];
    const bool stage = s_ok && row_hi - row_lo <= kCap;  // the same for every thread
    __syncthreads();  // the previous range's rows and labels are no longer read
    uint32_t extra = 0;  // words copied before row_lo (the copy starts on a 16-byte boundary)
    if (stage) {
      const uint64_t b_lo = static_cast<uint64_t>(row_lo) * AW * 8, b_hi = static_cast<uint64_t>(row_hi) * AW * 8;
      const uint64_t a_lo = b_lo & ~15ull;
      const uint64_t a_hi = (b_hi + 15) & ~15ull;
      const uint64_t c_hi = a_hi <= adj_bytes ? a_hi : (b_hi & ~15ull);  // the copy ends inside the array
      extra = static_cast<uint32_t>((b_lo - a_lo) / 8);
      if (threadIdx.x == 0) {
        if (c_hi > a_lo) {
          mbar_expect_tx(&s_bar, static_cast<uint32_t>(c_hi - a_lo));
          bulk_copy_g2s(s_rows, reinterpret_cast<const char*>(adj) + a_lo, static_cast<uint32_t>(c_hi - a_lo), &s_bar);
        } else {
          mbar_expect_tx(&s_bar, 0);  // completes the phase with nothing in flight
        }
      }
      if (threadIdx.x == 32 && c_hi < b_hi) {  // the last 8-byte row past the final 16-byte boundary
        s_rows[(c_hi - a_lo) / 8] = adj[(c_hi) / 8];
        // order this generic store before any later bulk copy into the buffer
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      }
      for (uint32_t i = threadIdx.x; i < row_hi - row_lo; i += blockDim.x) s_lab[i] = lab[row_lo + i];
      if (!mbar_wait(&s_bar, parity)) s_ok = 0;
      parity ^= 1u;
    }
    __syncthreads();  // labels and the tail row are in; s_ok is settled
    const bool use_smem = stage && s_ok;
    const uint64_t vv = v0 + threadIdx.x;
    if (vv >= v1) continue;
    const uint32_t v = static_cast<uint32_t>(vv);
    const uint32_t prev = goff[node_graph[v]];
    const uint32_t n = goff[node_graph[v] + 1] - prev;
    const uint32_t lv = v - prev;
    // rows and labels of this vertex's graph: shared memory or global memory
    const uint64_t* grow = use_smem ? s_rows + extra + static_cast<uint64_t>(prev - row_lo) * AW : adj + static_cast<uint64_t>(prev) * AW;
    const uint8_t* glab = use_smem ? s_lab + (prev - row_lo) : lab + prev;
    uint64_t F[AW], R[AW];
    const bool wide = !EXACT && n > 256u;
#pragma unroll
    for (int k = 0; k < AW; ++k) F[k] = 0;
    if (EXACT) {
#pragma unroll
      for (int k = 0; k < AW; ++k) F[k] = ((lv >> 6) == (uint32_t)k) ? (1ull << (lv & 63u)) : 0ull;
    } else {
      F[0] = wide ? refbit(lv, 0) : (lv < 64u ? (1ull << lv) : 0ull);
    }
#pragma unroll
    for (int k = 0; k < AW; ++k) R[k] = F[k];
    for (uint32_t r = 0; r < Rn; ++r) {
      uint64_t nx[AW];
#pragma unroll
      for (int k = 0; k < AW; ++k) nx[k] = 0;
      if (EXACT) {
#pragma unroll
        for (int w = 0; w < AW; ++w) {
          uint64_t m = F[w];
          while (m) {
            const uint32_t b = __ffsll(static_cast<long long>(m)) - 1 + 64u * w;
            m &= m - 1;
            const uint64_t* row = grow + static_cast<uint64_t>(b) * AW;
#pragma unroll
            for (int k = 0; k < AW; ++k) nx[k] |= row[k];
          }
        }
      } else {
        uint64_t m = F[0];
        while (m) {
          const uint32_t b = __ffsll(static_cast<long long>(m)) - 1;
          m &= m - 1;
          if (wide) {
            const uint32_t u = prev + b;
            for (uint32_t i = roff[u]; i < roff[u + 1]; ++i) nx[0] |= refbit(col[i] - prev, 0);
          } else {
            nx[0] |= grow[static_cast<uint64_t>(b) * AW];
          }
        }
      }
      uint64_t s = 0;
#pragma unroll
      for (int k = 0; k < AW; ++k) {
        nx[k] &= ~R[k];
        R[k] |= nx[k];
        F[k] = nx[k];
        uint64_t sphere = nx[k];
        while (sphere) {
          const uint32_t b = __ffsll(static_cast<long long>(sphere)) - 1;
          sphere &= sphere - 1;
          s = sig_inc(s, glab[64u * k + b]);
        }
        if (!EXACT) break;
      }
      sig_all[static_cast<uint64_t>(r) * N + v] = s;
    }
  }
  // a copy whose wait ran out may still be in flight: wait again (bounded)
  // before the CTA's shared memory is released
  __syncthreads();
  if (!s_ok) mbar_wait(&s_bar, parity ^ 1u);
}

// Matching order per query graph (batched join): start at the vertex of
// highest degree, then repeatedly take the vertex with the most neighbours
// already placed (ties: higher degree, lower id).  qorder[off + k] = local id
// placed at level k; qsel[off + k] = levels i < k adjacent to level k in that
// order; qsel_id[off + k] = the same for the identity order (used when a graph
// has an asymmetric adjacency, which only self-loops produce).  sym[g] = 1 if
// every adjacency row of graph g is mirrored.
__global__ void k_query_order(uint32_t QG, const uint32_t* __restrict__ goff, const uint64_t* __restrict__ adj,
                              uint8_t* __restrict__ qorder, uint64_t* __restrict__ qsel, uint64_t* __restrict__ qsel_id) {
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < QG; q += gridDim.x * blockDim.x) {
    const uint32_t off = goff[q], n = goff[q + 1] - off;
    if (n > kMaxQueryNodes) continue;
    uint64_t placed = 0;
    uint8_t ord[kMaxQueryNodes];
    for (uint32_t k = 0; k < n; ++k) {
      int best = -1, best_conn = -1, best_deg = -1;
      for (uint32_t u = 0; u < n; ++u) {
        if ((placed >> u) & 1ull) continue;
        const uint64_t row = adj[off + u];
        const int conn = __popcll(row & placed);
        const int deg = __popcll(row);
        if (conn > best_conn || (conn == best_conn && deg > best_deg)) {
          best = static_cast<int>(u);
          best_conn = conn;
          best_deg = deg;
        }
      }
      ord[k] = static_cast<uint8_t>(best);
      placed |= 1ull << best;
    }
    for (uint32_t k = 0; k < n; ++k) {
      uint64_t sel = 0, sel_id = 0;
      for (uint32_t i = 0; i < k; ++i) {
        if ((adj[off + ord[i]] >> ord[k]) & 1ull) sel |= 1ull << i;
        if ((adj[off + i] >> k) & 1ull) sel_id |= 1ull << i;
      }
      qorder[off + k] = ord[k];
      qsel[off + k] = sel;
      qsel_id[off + k] = sel_id;
    }
  }
}

template <int AW>
__global__ void k_graph_symmetric(uint32_t G, const uint32_t* __restrict__ goff, const uint64_t* __restrict__ adj,
                                  uint8_t* __restrict__ sym) {
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < G; g += gridDim.x * blockDim.x) {
    const uint32_t off = goff[g], n = goff[g + 1] - off;
    // mirrored iff every edge u -> t (t < n) has t -> u: a missing reverse
    // edge is found from the row that holds the edge, so only set bits are visited
    bool ok = n <= 64u * AW;
    for (uint32_t u = 0; u < n && ok; ++u)
      for (uint32_t w = 0; w < static_cast<uint32_t>(AW) && ok; ++w) {
        const uint32_t lo = 64u * w;
        uint64_t bits = lo < n ? adj[static_cast<uint64_t>(off + u) * AW + w] : 0ull;
        if (lo < n && n - lo < 64u) bits &= (1ull << (n - lo)) - 1ull;
        while (bits && ok) {
          const uint32_t t = lo + static_cast<uint32_t>(__ffsll(static_cast<long long>(bits))) - 1u;
          bits &= bits - 1;
          ok = (adj[static_cast<uint64_t>(off + t) * AW + (u >> 6)] >> (u & 63u)) & 1ull;
        }
      }
    sym[g] = ok ? 1 : 0;
  }
}

}  // namespace

int launch_graph_derive(Graph* g) {
  Queue* q = g->q;
  const unsigned B = 256;
  if (g->total_nodes) {
    SIGMO_TRY(dev_alloc(q, reinterpret_cast<void**>(&g->node_graph), sizeof(uint32_t) * g->total_nodes));
    k_node_graph<<<grid_for(g->num_graphs, B, 65535u), B, 0, q->stream>>>(g->graph_offsets, g->num_graphs, g->node_graph);
    SIGMO_TRY(check_launch(q, "k_node_graph"));
  }
  // words per local adjacency row: 1, 2 or 4 (the kernels are instantiated
  // for those widths; a batch whose largest graph has 129-192 vertices gets 4)
  const uint32_t mx = g->max_nodes;
  uint32_t aw = 1;
  while (aw < kMaxAdjWords && aw * 64u < mx) aw *= 2;
  g->adj_words = aw;
  const uint64_t adj_elems = g->total_nodes * aw;
  SIGMO_TRY(dev_alloc(q, reinterpret_cast<void**>(&g->adj), sizeof(uint64_t) * (adj_elems ? adj_elems : 1)));
  SIGMO_TRY(dev_alloc(q, reinterpret_cast<void**>(&g->sym), g->num_graphs ? g->num_graphs : 1));
  if (g->total_nodes) {
    const unsigned grid = grid_for(g->total_nodes, B, 148u * 32u);
    switch (aw) {
      case 1: k_build_adj<1><<<grid, B, 0, q->stream>>>(g->total_nodes, g->row_offsets, g->column_indices, g->graph_offsets, g->node_graph, g->adj); break;
      case 2: k_build_adj<2><<<grid, B, 0, q->stream>>>(g->total_nodes, g->row_offsets, g->column_indices, g->graph_offsets, g->node_graph, g->adj); break;
      default: k_build_adj<4><<<grid, B, 0, q->stream>>>(g->total_nodes, g->row_offsets, g->column_indices, g->graph_offsets, g->node_graph, g->adj); break;
    }
    SIGMO_TRY(check_launch(q, "k_build_adj"));
  }
  if (g->num_graphs) {
    const unsigned grid = grid_for(g->num_graphs, B, 148u * 32u);
    switch (aw) {
      case 1: k_graph_symmetric<1><<<grid, B, 0, q->stream>>>(g->num_graphs, g->graph_offsets, g->adj, g->sym); break;
      case 2: k_graph_symmetric<2><<<grid, B, 0, q->stream>>>(g->num_graphs, g->graph_offsets, g->adj, g->sym); break;
      default: k_graph_symmetric<4><<<grid, B, 0, q->stream>>>(g->num_graphs, g->graph_offsets, g->adj, g->sym); break;
    }
    SIGMO_TRY(check_launch(q, "k_graph_symmetric"));
  }
  return SIGMO_OK;
}

int launch_query_order(Graph* g) {
  Queue* q = g->q;
  if (g->qorder) return SIGMO_OK;
  SIGMO_TRY(dev_alloc(q, reinterpret_cast<void**>(&g->qorder), g->total_nodes ? g->total_nodes : 1));
  SIGMO_TRY(dev_alloc(q, reinterpret_cast<void**>(&g->qsel), sizeof(uint64_t) * (g->total_nodes ? g->total_nodes : 1)));
  SIGMO_TRY(dev_alloc(q, reinterpret_cast<void**>(&g->qsel_id), sizeof(uint64_t) * (g->total_nodes ? g->total_nodes : 1)));
  if (g->num_graphs && g->adj_words == 1) {
    k_query_order<<<grid_for(g->num_graphs, 128, 4096u), 128, 0, q->stream>>>(g->num_graphs, g->graph_offsets, g->adj,
                                                                               g->qorder, g->qsel, g->qsel_id);
    SIGMO_TRY(check_launch(q, "k_query_order"));
  }
  return SIGMO_OK;
}

int launch_sig_generate(Queue* q, const Graph* g, uint64_t* sig) {
  if (!g->total_nodes) return SIGMO_OK;
  k_sig_generate<<<grid_for(g->total_nodes, 256, 148u * 32u), 256, 0, q->stream>>>(g->total_nodes, g->row_offsets,
                                                                                   g->column_indices, g->node_labels, sig);
  return check_launch(q, "k_sig_generate");
}

int launch_sig_refine(Queue* q, const Graph* g, uint32_t view, uint64_t* sig, uint64_t* reach, uint32_t reach_words) {
  if (!g->total_nodes) return SIGMO_OK;
  const unsigned grid = grid_for(g->total_nodes, 256, 148u * 32u);
  if (q->opts.profile == kProfileExact) {
    if (g->max_nodes > 64u * kMaxAdjWords)
      return fail(SIGMO_ERR_DOMAIN, "exact profile supports graphs of at most %u vertices (largest: %u)", 64u * kMaxAdjWords, g->max_nodes);
    if (reach_words != kMaxAdjWords) return fail(SIGMO_ERR_INVALID, "exact profile needs %u reachable words", kMaxAdjWords);
    switch (g->adj_words) {
      case 1: k_sig_refine_exact<1><<<grid, 256, 0, q->stream>>>(g->total_nodes, g->graph_offsets, g->node_graph, g->adj, g->node_labels, view, sig, reach); break;
      case 2: k_sig_refine_exact<2><<<grid, 256, 0, q->stream>>>(g->total_nodes, g->graph_offsets, g->node_graph, g->adj, g->node_labels, view, sig, reach); break;
      default: k_sig_refine_exact<4><<<grid, 256, 0, q->stream>>>(g->total_nodes, g->graph_offsets, g->node_graph, g->adj, g->node_labels, view, sig, reach); break;
    }
    return check_launch(q, "k_sig_refine_exact");
  }
  if (q->opts.profile == kProfileX86) {
    if (g->max_nodes > 64u * kMaxAdjWords)
      return fail(SIGMO_ERR_DOMAIN, "REF_X86 profile supports graphs of at most %u vertices (largest: %u)", 64u * kMaxAdjWords,
                  g->max_nodes);
    k_sig_refine_ptx<true><<<grid, 256, 0, q->stream>>>(g->total_nodes, g->graph_offsets, g->node_graph, g->adj, g->adj_words,
                                                        g->row_offsets, g->column_indices, g->node_labels, view, sig, reach);
    return check_launch(q, "k_sig_refine_x86");
  }
  k_sig_refine_ptx<false><<<grid, 256, 0, q->stream>>>(g->total_nodes, g->graph_offsets, g->node_graph, g->adj, g->adj_words,
                                                       g->row_offsets, g->column_indices, g->node_labels, view, sig, reach);
  return check_launch(q, "k_sig_refine_ptx");
}

int launch_sig_all(Queue* q, const Graph* g, uint32_t R, uint64_t* sig_all) {
  if (!g->total_nodes || !R) return SIGMO_OK;
  const unsigned grid = grid_for(g->total_nodes, 256, 148u * 32u);
  if (q->opts.profile == kProfileExact) {
    if (g->max_nodes > 64u * kMaxAdjWords)
      return fail(SIGMO_ERR_DOMAIN, "exact profile supports graphs of at most %u vertices (largest: %u)", 64u * kMaxAdjWords, g->max_nodes);
    switch (g->adj_words) {
      case 1: k_sig_all_staged<1, true><<<grid, kSigRange, 0, q->stream>>>(g->total_nodes, g->graph_offsets, g->node_graph, g->adj, g->row_offsets, g->column_indices, g->node_labels, R, sig_all); break;
      case 2: k_sig_all_staged<2, true><<<grid, kSigRange, 0, q->stream>>>(g->total_nodes, g->graph_offsets, g->node_graph, g->adj, g->row_offsets, g->column_indices, g->node_labels, R, sig_all); break;
      default: k_sig_all_staged<4, true><<<grid, kSigRange, 0, q->stream>>>(g->total_nodes, g->graph_offsets, g->node_graph, g->adj, g->row_offsets, g->column_indices, g->node_labels, R, sig_all); break;
    }
    return check_launch(q, "k_sig_all<exact>");
  }
  switch (g->adj_words) {
    case 1: k_sig_all_staged<1, false><<<grid, kSigRange, 0, q->stream>>>(g->total_nodes, g->graph_offsets, g->node_graph, g->adj, g->row_offsets, g->column_indices, g->node_labels, R, sig_all); break;
    case 2: k_sig_all_staged<2, false><<<grid, kSigRange, 0, q->stream>>>(g->total_nodes, g->graph_offsets, g->node_graph, g->adj, g->row_offsets, g->column_indices, g->node_labels, R, sig_all); break;
    default: k_sig_all_staged<4, false><<<grid, kSigRange, 0, q->stream>>>(g->total_nodes, g->graph_offsets, g->node_graph, g->adj, g->row_offsets, g->column_indices, g->node_labels, R, sig_all); break;
  }
  return check_launch(q, "k_sig_all<ptx>");
}

}  // namespace sigmo_b200
