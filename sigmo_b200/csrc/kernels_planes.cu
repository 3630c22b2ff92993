// Batched form: per-graph candidate planes.
//
// The reference's candidate test for query vertex j and data vertex d after
// R refinements is (isomorphism.hpp:48-55, 103-111)
//     label(j) == label(d) (or label(j) is the wildcard)
//     and, for every iteration r and label l, count_l(sig_r(j)) <= count_l(sig_r(d)).
// For a fixed query batch the set of thresholds that appear is small, so each
// data graph gets one u64 mask ("plane") per distinct query label and per
// distinct (r, l, c) threshold: bit t = local vertex t passes.  The candidate
// set of query vertex j in data graph g is then the AND of the planes in j's
// program; graph-local range visibility (the REF_PTX last-word rule of
// candidates.hpp:98) is folded into the label planes.  Identical query
// vertices share one program ("class").
//
// Plane layout: planes[((g / 32) * K + k) * AW + w][g % 32] (u64), so the
// planes of 32 consecutive graphs form one contiguous tile that a CTA copies
// to shared memory and reads with lane = graph, conflict-free.
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.hpp"

namespace sigmo_b200 {
namespace {

// spec[k]: bit 31 set = label plane (bits 0..7 = label value, 255 = any);
// otherwise r = bits 16..23, l = bits 8..15, c = bits 0..7 (count >= c).

// Warp per data graph; lanes hold vertices lane + 32 p.
template <int AW>
__global__ void __launch_bounds__(256) k_build_planes(uint32_t G, const uint32_t* __restrict__ goff,
                                                     const uint8_t* __restrict__ lab, const uint64_t* __restrict__ sig_all,
                                                     uint64_t N, uint32_t R, uint32_t K, const uint32_t* __restrict__ spec,
                                                     int prof, uint64_t* __restrict__ planes) {
  constexpr int P = 2 * AW;  // 32-vertex chunks per graph
  const unsigned lane = threadIdx.x & 31u;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t g = warp; g < G; g += nwarps) {
    const uint32_t s = goff[g], e = goff[g + 1], n = e - s;
    uint8_t lb[P];
    bool vis[P];
    uint64_t sg[P][8];  // iterations beyond 8 are re-read from memory
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const uint32_t t = lane + 32u * p;
      const bool in = t < n;
      const uint32_t v = s + t;
      lb[p] = in ? lab[v] : 0;
      vis[p] = in && ((range_mask(v >> 5, s, e, prof) >> (v & 31u)) & 1u);
#pragma unroll
      for (int r = 0; r < 8; ++r) sg[p][r] = (in && static_cast<uint32_t>(r) < R) ? sig_all[static_cast<uint64_t>(r) * N + v] : 0ull;
    }
    uint64_t* out = planes + static_cast<uint64_t>(g >> 5) * K * AW * 32 + (g & 31u);
    for (uint32_t k = 0; k < K; ++k) {
      const uint32_t sp = spec[k];
      const bool is_label = (sp & 0x80000000u) != 0;
      const uint32_t r = (sp >> 16) & 0xFFu, l = (sp >> 8) & 0xFFu, c = sp & 0xFFu;
      uint32_t chunk[P];
#pragma unroll
      for (int p = 0; p < P; ++p) {
        bool pred;
        if (is_label) {
          const uint32_t val = sp & 0xFFu;
          pred = vis[p] && (val == kWildcard || lb[p] == val);
        } else {
          uint64_t sv = 0;
          const uint32_t t = lane + 32u * p;
          if (r < 8) {
#pragma unroll
            for (int rr = 0; rr < 8; ++rr)
              if (static_cast<uint32_t>(rr) == r) sv = sg[p][rr];
          } else if (t < n && r < R) {
            sv = sig_all[static_cast<uint64_t>(r) * N + s + t];
          }
          pred = t < n && r < R && sig_get(sv, l) >= c;
        }
        chunk[p] = __ballot_sync(0xFFFFFFFFu, pred);
      }
#pragma unroll
      for (int w = 0; w < AW; ++w) {
        const uint64_t word = static_cast<uint64_t>(chunk[2 * w]) | (static_cast<uint64_t>(chunk[2 * w + 1]) << 32);
        if (lane == ((k * AW + w) & 31u)) out[(static_cast<uint64_t>(k) * AW + w) * 32] = word;
      }
    }
  }
}

// NE[class][g/32]: bit = the class's candidate set in data graph g is non-empty.
// CTA per 32-graph tile; the tile's planes are staged in shared memory.
template <int AW>
__global__ void __launch_bounds__(256) k_ne_planes(const uint64_t* __restrict__ planes, uint32_t K, uint32_t GW,
                                                  uint32_t C, const uint32_t* __restrict__ prog_off,
                                                  const uint16_t* __restrict__ prog, uint32_t* __restrict__ NE) {
  extern __shared__ uint64_t tile[];  // [K * AW][32]
  const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (uint32_t gw = blockIdx.x; gw < GW; gw += gridDim.x) {
    __syncthreads();
    const uint4* src = reinterpret_cast<const uint4*>(planes + static_cast<uint64_t>(gw) * K * AW * 32);
    uint4* dst = reinterpret_cast<uint4*>(tile);
    const uint32_t n16 = K * AW * 16;  // uint4 per tile
    for (uint32_t i = threadIdx.x; i < n16; i += blockDim.x) dst[i] = __ldg(src + i);
    __syncthreads();
    for (uint32_t c = wid; c < C; c += nw) {
      uint64_t m[AW];
#pragma unroll
      for (int w = 0; w < AW; ++w) m[w] = ~0ull;
      const uint32_t e0 = prog_off[c], e1 = prog_off[c + 1];
      for (uint32_t e = e0; e < e1; ++e) {
        const uint32_t k = prog[e];
#pragma unroll
        for (int w = 0; w < AW; ++w) m[w] &= tile[(k * AW + w) * 32 + lane];
        if (((e - e0) & 3u) == 3u) {
          bool any = false;
#pragma unroll
          for (int w = 0; w < AW; ++w) any |= m[w] != 0;
          if (!__any_sync(0xFFFFFFFFu, any)) break;
        }
      }
      bool any = false;
#pragma unroll
      for (int w = 0; w < AW; ++w) any |= m[w] != 0;
      const uint32_t word = __ballot_sync(0xFFFFFFFFu, any);
      if (lane == 0) NE[static_cast<uint64_t>(c) * GW + gw] = word;
    }
  }
}

}  // namespace

int launch_build_planes(Queue* q, const Graph* data, const uint64_t* sig_all, uint32_t R, const PlaneProgram& pp,
                        uint64_t* planes) {
  if (!data->num_graphs) return SIGMO_OK;
  const unsigned block = 256;
  const unsigned grid = grid_for(static_cast<uint64_t>(data->num_graphs) * 32, block, 148u * 16u);
  switch (data->adj_words) {
    case 1: k_build_planes<1><<<grid, block, 0, q->stream>>>(data->num_graphs, data->graph_offsets, data->node_labels, sig_all, data->total_nodes, R, pp.K, pp.spec, q->opts.profile, planes); break;
    case 2: k_build_planes<2><<<grid, block, 0, q->stream>>>(data->num_graphs, data->graph_offsets, data->node_labels, sig_all, data->total_nodes, R, pp.K, pp.spec, q->opts.profile, planes); break;
    default: k_build_planes<4><<<grid, block, 0, q->stream>>>(data->num_graphs, data->graph_offsets, data->node_labels, sig_all, data->total_nodes, R, pp.K, pp.spec, q->opts.profile, planes); break;
  }
  return check_launch(q, "k_build_planes");
}

size_t ne_planes_smem(uint32_t K, uint32_t AW) { return static_cast<size_t>(K) * AW * 32 * 8; }

int launch_ne_planes(Queue* q, const Graph* data, const PlaneProgram& pp, const uint64_t* planes, uint32_t* NE) {
  const uint32_t GW = (data->num_graphs + 31u) / 32u;
  if (!GW || !pp.C) return SIGMO_OK;
  const size_t smem = ne_planes_smem(pp.K, data->adj_words);
  const unsigned block = 256;
  const unsigned grid = std::min<uint32_t>(GW, 148u * 8u);
  cudaError_t e = cudaSuccess;
  switch (data->adj_words) {
    case 1:
      e = cudaFuncSetAttribute(k_ne_planes<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
      if (e == cudaSuccess) k_ne_planes<1><<<grid, block, smem, q->stream>>>(planes, pp.K, GW, pp.C, pp.prog_off, pp.prog, NE);
      break;
    case 2:
      e = cudaFuncSetAttribute(k_ne_planes<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
      if (e == cudaSuccess) k_ne_planes<2><<<grid, block, smem, q->stream>>>(planes, pp.K, GW, pp.C, pp.prog_off, pp.prog, NE);
      break;
    default:
      e = cudaFuncSetAttribute(k_ne_planes<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
      if (e == cudaSuccess) k_ne_planes<4><<<grid, block, smem, q->stream>>>(planes, pp.K, GW, pp.C, pp.prog_off, pp.prog, NE);
      break;
  }
  if (e != cudaSuccess) return fail(SIGMO_ERR_CUDA, "k_ne_planes shared-memory setup failed: %s", cudaGetErrorString(e));
  return check_launch(q, "k_ne_planes");
}

}  // namespace sigmo_b200
