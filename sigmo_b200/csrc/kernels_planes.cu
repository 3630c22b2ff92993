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

// One graph's planes into column `gl` of a shared-memory tile [K * AW][32]:
// the warp's lanes hold vertices lane + 32 p, every plane is a ballot per
// 32-vertex chunk, and the plane word is stored by a single lane.
template <int AW>
__device__ __forceinline__ void build_graph_planes(uint64_t* tile, uint32_t gl, uint32_t s, uint32_t e, unsigned lane,
                                                   const uint8_t* __restrict__ lab, const uint64_t* __restrict__ sig_all,
                                                   uint64_t N, uint32_t R, uint32_t K, const uint32_t* __restrict__ spec,
                                                   int prof) {
  constexpr int P = 2 * AW;  // 32-vertex chunks per graph
  const uint32_t n = e - s;
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
  for (uint32_t k = 0; k < K; ++k) {
    const uint32_t sp = spec[k];
    const bool is_label = (sp & 0x80000000u) != 0;
    const uint32_t r = (sp >> 16) & 0xFFu, l = (sp >> 8) & 0xFFu, c = sp & 0xFFu;
    uint32_t chunk[P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      bool pred;
      const uint32_t t = lane + 32u * p;
      if (is_label) {
        const uint32_t val = sp & 0xFFu;
        pred = vis[p] && (val == kWildcard || lb[p] == val);
      } else {
        uint64_t sv = 0;
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
      if (lane == ((k * AW + w) & 31u)) tile[(k * AW + w) * 32 + gl] = word;
    }
  }
}

// Per 32-graph tile (one CTA per tile, grid-stride): build the tile's planes
// in shared memory from the data signatures, write the tile out (coalesced;
// the join reads it), then NE[class][tile] = ballot over the tile's graphs of
// "AND of the class's program planes != 0".  Classes are numbered in
// lexicographic program order and each warp walks a contiguous class range
// keeping the running prefix ANDs (depth < kPrefix) in shared memory, so a
// class only ANDs the part of its program it does not share with its
// predecessor, and a prefix that is empty for all 32 graphs ends every class
// below it at once.
constexpr uint32_t kPrefix = 16;

template <int AW>
__global__ void __launch_bounds__(256) k_planes_ne(uint32_t G, const uint32_t* __restrict__ goff, const uint8_t* __restrict__ lab,
                                                  const uint64_t* __restrict__ sig_all, uint64_t N, uint32_t R, uint32_t K,
                                                  const uint32_t* __restrict__ spec, int prof, uint32_t C,
                                                  const uint32_t* __restrict__ prog_off, const uint16_t* __restrict__ prog,
                                                  const uint8_t* __restrict__ cp, uint64_t* __restrict__ planes,
                                                  uint32_t* __restrict__ NE) {
  extern __shared__ uint64_t tile[];  // [K * AW][32], then prefix stacks [8 warps][kPrefix][AW][32]
  const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint32_t GW = (G + 31u) / 32u;
  const uint32_t words = K * AW;
  uint64_t* pst = tile + static_cast<size_t>(words) * 32 + static_cast<size_t>(wid) * kPrefix * AW * 32;
  const uint32_t per_warp = (C + nw - 1) / nw;
  const uint32_t c_begin = wid * per_warp, c_end = c_begin + per_warp < C ? c_begin + per_warp : C;
  for (uint32_t gw = blockIdx.x; gw < GW; gw += gridDim.x) {
    __syncthreads();  // the previous tile is no longer read
    for (uint32_t gl = wid; gl < 32; gl += nw) {
      const uint32_t g = gw * 32u + gl;
      if (g < G) {
        build_graph_planes<AW>(tile, gl, goff[g], goff[g + 1], lane, lab, sig_all, N, R, K, spec, prof);
      } else {
        for (uint32_t i = lane; i < words; i += 32) tile[i * 32 + gl] = 0;
      }
    }
    __syncthreads();
    {
      uint4* dst = reinterpret_cast<uint4*>(planes + static_cast<uint64_t>(gw) * words * 32);
      const uint4* src = reinterpret_cast<const uint4*>(tile);
      for (uint32_t i = threadIdx.x; i < words * 16; i += blockDim.x) dst[i] = src[i];
    }
    uint32_t valid = 0;  // prefix depths held in pst from the previous class
    for (uint32_t c = c_begin; c < c_end; ++c) {
      const uint32_t e0 = prog_off[c], len = prog_off[c + 1] - e0;
      uint32_t d = c == c_begin ? 0u : min(static_cast<uint32_t>(cp[c]), valid);
      uint64_t m[AW];
#pragma unroll
      for (int w = 0; w < AW; ++w) m[w] = d ? pst[((d - 1) * AW + w) * 32 + lane] : ~0ull;
      bool alive;
      {
        bool any = false;
#pragma unroll
        for (int w = 0; w < AW; ++w) any |= m[w] != 0;
        alive = __any_sync(0xFFFFFFFFu, any);
      }
      uint32_t reached = d;
      for (; d < len && alive; ++d) {
        const uint32_t k = prog[e0 + d];
        bool any = false;
#pragma unroll
        for (int w = 0; w < AW; ++w) {
          m[w] &= tile[(k * AW + w) * 32 + lane];
          any |= m[w] != 0;
        }
        if (d < kPrefix) {
#pragma unroll
          for (int w = 0; w < AW; ++w) pst[(d * AW + w) * 32 + lane] = m[w];
        }
        reached = d + 1;
        alive = __any_sync(0xFFFFFFFFu, any);
      }
      valid = reached < kPrefix ? reached : kPrefix;
      bool any = false;
#pragma unroll
      for (int w = 0; w < AW; ++w) any |= m[w] != 0;
      const uint32_t word = __ballot_sync(0xFFFFFFFFu, alive && any);
      if (lane == 0) NE[static_cast<uint64_t>(c) * GW + gw] = word;
    }
  }
}

}  // namespace

size_t ne_planes_smem(uint32_t K, uint32_t AW) {
  return static_cast<size_t>(K) * AW * 32 * 8 + static_cast<size_t>(8) * kPrefix * AW * 32 * 8;
}

int launch_planes_ne(Queue* q, const Graph* data, const uint64_t* sig_all, uint32_t R, const PlaneProgram& pp,
                     uint64_t* planes, uint32_t* NE) {
  const uint32_t G = data->num_graphs, GW = (G + 31u) / 32u;
  if (!GW) return SIGMO_OK;
  const size_t smem = ne_planes_smem(pp.K, data->adj_words);
  const unsigned block = 256;
  const unsigned grid = std::min<uint32_t>(GW, 148u * 8u);
  cudaError_t e = cudaSuccess;
#define SIGMO_PLANES_NE(AWV)                                                                                             \
  e = cudaFuncSetAttribute(k_planes_ne<AWV>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));      \
  if (e == cudaSuccess)                                                                                                  \
    k_planes_ne<AWV><<<grid, block, smem, q->stream>>>(G, data->graph_offsets, data->node_labels, sig_all,              \
                                                      data->total_nodes, R, pp.K, pp.spec, q->opts.profile, pp.C,      \
                                                      pp.prog_off, pp.prog, pp.cp, planes, NE)
  switch (data->adj_words) {
    case 1: SIGMO_PLANES_NE(1); break;
    case 2: SIGMO_PLANES_NE(2); break;
    default: SIGMO_PLANES_NE(4); break;
  }
#undef SIGMO_PLANES_NE
  if (e != cudaSuccess) return fail(SIGMO_ERR_CUDA, "k_planes_ne shared-memory setup failed: %s", cudaGetErrorString(e));
  return check_launch(q, "k_planes_ne");
}

}  // namespace sigmo_b200
