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
// Label planes come first, then thresholds in (r, l, c) order;
// r_begin[r] .. r_begin[r + 1] are the thresholds of iteration r.

// One graph's planes into column `gl` of a shared-memory tile [K * AW][32]:
// the warp's lanes hold vertices lane + 32 p, every plane is a ballot per
// 32-vertex chunk, and the plane word is stored by a single lane.  Chunks
// beyond the graph's last vertex are skipped (the warp handles one graph, so
// that test is uniform).
template <int AW>
__device__ __forceinline__ void build_graph_planes(uint64_t* tile, uint32_t gl, uint32_t s, uint32_t e, unsigned lane,
                                                   const uint8_t* __restrict__ lab, const uint64_t* __restrict__ sig_all,
                                                   uint64_t N, uint32_t R, uint32_t nlab, const uint32_t* __restrict__ spec,
                                                   const uint32_t* __restrict__ r_begin, int prof) {
  constexpr int P = 2 * AW;  // 32-vertex chunks per graph
  const uint32_t n = e - s;
  const uint32_t chunks = (n + 31u) / 32u;
  uint8_t lb[P];
  bool vis[P];
#pragma unroll
  for (int p = 0; p < P; ++p) {
    const uint32_t t = lane + 32u * p;
    const bool in = t < n;
    const uint32_t v = s + t;
    lb[p] = in ? lab[v] : 0;
    vis[p] = in && ((range_mask(v >> 5, s, e, prof) >> (v & 31u)) & 1u);
  }
  auto put = [&](uint32_t k, const uint32_t (&chunk)[P]) {
#pragma unroll
    for (int w = 0; w < AW; ++w) {
      const uint64_t word = static_cast<uint64_t>(chunk[2 * w]) | (static_cast<uint64_t>(chunk[2 * w + 1]) << 32);
      if (lane == ((k * AW + w) & 31u)) tile[(k * AW + w) * 32 + gl] = word;
    }
  };
  for (uint32_t k = 0; k < nlab; ++k) {
    const uint32_t val = spec[k] & 0xFFu;
    uint32_t chunk[P];
#pragma unroll
    for (int p = 0; p < P; ++p)
      chunk[p] = static_cast<uint32_t>(p) < chunks ? __ballot_sync(0xFFFFFFFFu, vis[p] && (val == kWildcard || lb[p] == val)) : 0u;
    put(k, chunk);
  }
  for (uint32_t r = 0; r < R; ++r) {
    const uint32_t k0 = r_begin[r], k1 = r_begin[r + 1];
    if (k0 == k1) continue;
    uint64_t sg[P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const uint32_t t = lane + 32u * p;
      sg[p] = (static_cast<uint32_t>(p) < chunks && t < n) ? sig_all[static_cast<uint64_t>(r) * N + s + t] : 0ull;
    }
    for (uint32_t k = k0; k < k1; ++k) {
      const uint32_t sp = spec[k];
      const uint32_t sh = 4u * ((sp >> 8) & 0xFFu), c = sp & 0xFFu;
      uint32_t chunk[P];
#pragma unroll
      for (int p = 0; p < P; ++p)
        chunk[p] = static_cast<uint32_t>(p) < chunks
                       ? __ballot_sync(0xFFFFFFFFu, static_cast<uint32_t>((sg[p] >> sh) & 0xFull) >= c)
                       : 0u;
      put(k, chunk);
    }
  }
}

// Per 32-graph tile (one CTA per tile, grid-stride): build the tile's planes
// in shared memory from the data signatures, write the tile out (coalesced;
// the join reads it), then walk the trie of the class programs:
// NE[class][tile] = ballot over the tile's graphs of "AND of the class's
// program planes != 0".
//
// The trie (host-built, preorder) stores per node a uint4 {x, skip, class, y}:
//   x bits 0..19  the node's plane (row index in the tile)
//     bit  20     the parent mask is read from the stack (else it is the
//                 previous node's mask, kept in registers)
//     bit  21     branch node (two or more children): save the mask
//     bit  22     terminal: `class` is the class whose program ends here
//   y bits 0..15  stack slot to read the parent mask from
//     bits 16..31 stack slot to save this node's mask to
//   skip          the preorder index after this node's subtree
// A node whose mask is zero in all 32 graphs jumps to `skip`, so every class
// below a dead prefix is skipped (NE is zeroed beforehand).  A branch node's
// slot is its number of branch ancestors, so a saved mask is never
// overwritten while its later children can still read it; the last slot
// holds all ones and is the parent of the top-level nodes.
//
// The walk is split into segments starting at nodes of depth <= 1 (seg =
// {begin, end, z}); warps take segments of the tile from a shared counter.
// A segment starting at depth 1 first evaluates its parent, a top-level
// plane (z bit 31; z bits 0..19 its row, z bit 21 save it to slot 0).
// Each warp keeps a 32-node window of the trie in registers (one coalesced
// 16-byte load per lane) and reads it by shuffle.
constexpr uint32_t kWalkWarps = 16;
constexpr uint32_t kNodeStackRead = 1u << 20, kNodeBranch = 1u << 21, kNodeTerminal = 1u << 22;
constexpr uint32_t kNodeOffset = (1u << 20) - 1u;

template <int AW>
__global__ void __launch_bounds__(kWalkWarps * 32) k_planes_ne(
    uint32_t G, const uint32_t* __restrict__ goff, const uint8_t* __restrict__ lab, const uint64_t* __restrict__ sig_all,
    uint64_t N, uint32_t R, uint32_t K, uint32_t nlab, const uint32_t* __restrict__ spec, const uint32_t* __restrict__ r_begin,
    int prof, const uint4* __restrict__ trie, uint32_t trie_n, const uint4* __restrict__ segs, uint32_t nsegs,
    uint32_t nslots, uint64_t* __restrict__ planes, uint32_t* __restrict__ NE) {
  extern __shared__ uint64_t tile[];  // [K * AW][32], then stacks [kWalkWarps][nslots][AW][32]
  __shared__ uint32_t seg_next;
  constexpr uint32_t kRow = AW * 32u;  // u64 words per plane row or stack slot
  const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint32_t GW = (G + 31u) / 32u;
  const uint32_t words = K * AW;
  const uint64_t* tl = tile + lane;  // tl[offset + 32 w]: word w of this lane's graph
  uint64_t* sl = tile + static_cast<size_t>(words) * 32 + static_cast<size_t>(wid) * nslots * AW * 32 + lane;
#pragma unroll
  for (int w = 0; w < AW; ++w) sl[((nslots - 1) * AW + w) * 32] = ~0ull;  // the root slot
  for (uint32_t gw = blockIdx.x; gw < GW; gw += gridDim.x) {
    __syncthreads();  // the previous tile is no longer read
    for (uint32_t gl = wid; gl < 32; gl += nw) {
      const uint32_t g = gw * 32u + gl;
      if (g < G) {
        build_graph_planes<AW>(tile, gl, goff[g], goff[g + 1], lane, lab, sig_all, N, R, nlab, spec, r_begin, prof);
      } else {
        for (uint32_t i = lane; i < words; i += 32) tile[i * 32 + gl] = 0;
      }
    }
    if (threadIdx.x == 0) seg_next = 0;
    __syncthreads();
    {
      uint4* dst = reinterpret_cast<uint4*>(planes + static_cast<uint64_t>(gw) * words * 32);
      const uint4* src = reinterpret_cast<const uint4*>(tile);
      for (uint32_t i = threadIdx.x; i < words * 16; i += blockDim.x) dst[i] = src[i];
    }
    for (;;) {
      uint32_t si = 0;
      if (lane == 0) si = atomicAdd(&seg_next, 1u);
      si = __shfl_sync(0xFFFFFFFFu, si, 0);
      if (si >= nsegs) break;
      const uint4 sg = segs[si];
      uint64_t m[AW];
#pragma unroll
      for (int w = 0; w < AW; ++w) m[w] = ~0ull;
      if (sg.z & 0x80000000u) {  // the segment starts below a top-level node: evaluate it
#pragma unroll
        for (int w = 0; w < AW; ++w) {
          m[w] = tl[(sg.z & kNodeOffset) * kRow + 32 * w];
          if (sg.z & kNodeBranch) sl[32 * w] = m[w];  // slot 0
        }
      }
      uint32_t i = sg.x, wbase = 0xFFFFFFFFu;
      uint4 win = make_uint4(0, 0, 0, 0);
      while (i < sg.y) {
        if (i < wbase || i - wbase >= 32u) {
          wbase = i;
          win = i + lane < trie_n ? trie[i + lane] : make_uint4(0, 0, 0, 0);
        }
        const uint32_t at = i - wbase;
        const uint32_t x = __shfl_sync(0xFFFFFFFFu, win.x, at);
        const uint32_t y = __shfl_sync(0xFFFFFFFFu, win.w, at);
        const uint32_t off = (x & kNodeOffset) * kRow;
        bool any = false;
        if (x & kNodeStackRead) {
#pragma unroll
          for (int w = 0; w < AW; ++w) {
            m[w] = sl[(y & 0xFFFFu) * kRow + 32 * w] & tl[off + 32 * w];
            any |= m[w] != 0;
          }
        } else {
#pragma unroll
          for (int w = 0; w < AW; ++w) {
            m[w] &= tl[off + 32 * w];
            any |= m[w] != 0;
          }
        }
        if (!__any_sync(0xFFFFFFFFu, any)) {
          i = __shfl_sync(0xFFFFFFFFu, win.y, at);  // past this node's subtree
          continue;
        }
        if (x & kNodeBranch) {
#pragma unroll
          for (int w = 0; w < AW; ++w) sl[(y >> 16) * kRow + 32 * w] = m[w];
        }
        if (x & kNodeTerminal) {
          const uint32_t cls = __shfl_sync(0xFFFFFFFFu, win.z, at);
          const uint32_t word = __ballot_sync(0xFFFFFFFFu, any);
          if (lane == 0) NE[static_cast<uint64_t>(cls) * GW + gw] = word;
        }
        ++i;
      }
    }
  }
}

}  // namespace

size_t ne_planes_smem(uint32_t K, uint32_t AW, uint32_t nslots) {
  return static_cast<size_t>(K) * AW * 32 * 8 + static_cast<size_t>(kWalkWarps) * nslots * AW * 32 * 8;
}

int launch_planes_ne(Queue* q, const Graph* data, const uint64_t* sig_all, uint32_t R, const PlaneProgram& pp,
                     uint64_t* planes, uint32_t* NE) {
  const uint32_t G = data->num_graphs, GW = (G + 31u) / 32u;
  if (!GW) return SIGMO_OK;
  SIGMO_CUDA_TRY(cudaMemsetAsync(NE, 0, 4ull * pp.C * GW, q->stream));
  const size_t smem = ne_planes_smem(pp.K, data->adj_words, pp.nslots);
  const unsigned block = 32u * kWalkWarps;
  cudaError_t e = cudaSuccess;
  int per_sm = 0, sms = 0;
  SIGMO_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, q->device));
#define SIGMO_PLANES_NE(AWV)                                                                                          \
  e = cudaFuncSetAttribute(k_planes_ne<AWV>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));   \
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_planes_ne<AWV>, block, smem);    \
  if (e == cudaSuccess)                                                                                               \
    k_planes_ne<AWV><<<std::min<uint64_t>(GW, static_cast<uint64_t>(std::max(per_sm, 1)) * sms), block, smem,          \
                       q->stream>>>(G, data->graph_offsets, data->node_labels, sig_all, data->total_nodes, R, pp.K,   \
                                    pp.nlab, pp.spec, pp.r_begin, q->opts.profile, pp.trie, pp.trie_n, pp.segs,       \
                                    pp.nsegs, pp.nslots, planes, NE)
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
