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
                                                   const uint32_t* __restrict__ r_begin, int prof, uint32_t base) {
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
    // visibility follows global ids (base + local id): the range-mask rule
    // depends on where the graph ends relative to 32-vertex words
    const uint32_t gv = base + v;
    vis[p] = in && ((range_mask(gv >> 5, base + s, base + e, prof) >> (gv & 31u)) & 1u);
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
// the join reads it), then decide the GMCR admission of every query graph
// for the tile's 32 graphs (gmcr.hpp:33-128: every query vertex has a
// candidate in the graph):
//     admit[q][tile] = AND over q's classes c of NE(c),
//     NE(c) = ballot over the tile's graphs of "AND of c's program planes != 0".
// Warps take query graphs; a query's classes are visited in the order the
// host chose (rarest label first, longer programs first), so most queries
// are rejected for all 32 graphs after one or two classes and stop there.
// A class's AND chain stops as soon as it is zero in all 32 graphs.  NE(c)
// is evaluated for each query that reaches it: classes are rarely shared
// between queries, and without a per-class cache in shared memory four CTAs
// fit on an SM instead of three.  The per-graph admitted counts (the GMCR
// segment lengths) are summed in shared memory.  Queries of one vertex are
// never admitted (the reference's mapping skips them, gmcr.hpp:100): their
// class lists are empty.
constexpr uint32_t kAdmitWarps = 16;

// The tile's planes: built from the data signatures (and written out for the
// join), or gathered from resident planes (rows row_map[k] of the tile).
template <int AW, bool GATHER>
__device__ __forceinline__ void fill_tile(uint64_t* tile, uint32_t gw, uint32_t G, const uint32_t* __restrict__ goff,
                                          const uint8_t* __restrict__ lab, const uint64_t* __restrict__ sig_all, uint64_t N,
                                          uint32_t R, uint32_t K, uint32_t nlab, const uint32_t* __restrict__ spec,
                                          const uint32_t* __restrict__ r_begin, int prof, uint32_t base,
                                          const uint64_t* __restrict__ rplanes, uint32_t rrows,
                                          const uint32_t* __restrict__ row_map) {
  constexpr uint32_t kRow = AW * 32u;
  const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (GATHER) {
    const uint64_t* src = rplanes + static_cast<uint64_t>(gw) * rrows * kRow;
    for (uint32_t k = wid; k < K; k += nw) {
      const uint64_t* row = src + static_cast<uint64_t>(row_map[k]) * kRow;
#pragma unroll
      for (int w = 0; w < AW; ++w) tile[k * kRow + 32 * w + lane] = row[32 * w + lane];
    }
  } else {
    for (uint32_t gl = wid; gl < 32; gl += nw) {
      const uint32_t g = gw * 32u + gl;
      if (g < G) {
        build_graph_planes<AW>(tile, gl, goff[g], goff[g + 1], lane, lab, sig_all, N, R, nlab, spec, r_begin, prof, base);
      } else {
        for (uint32_t i = lane; i < K * AW; i += 32) tile[i * 32 + gl] = 0;
      }
    }
  }
}

// 16-byte asynchronous global -> shared copies (no registers in between).
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Resident rows row_map[k] of tile gw into dst (K rows of AW x 32 words),
// as 16-byte asynchronous copies spread over the block.
template <int AW>
__device__ __forceinline__ void gather_tile_async(uint64_t* dst, const uint64_t* __restrict__ rplanes, uint32_t rrows,
                                                  uint32_t gw, uint32_t K, const uint32_t* s_map) {
  constexpr uint32_t kRow = AW * 32u, kChunks = AW * 16u;  // 16-byte chunks per row
  const uint64_t* src = rplanes + static_cast<uint64_t>(gw) * rrows * kRow;
  for (uint32_t i = threadIdx.x; i < K * kChunks; i += blockDim.x) {
    const uint32_t k = i / kChunks, c = i % kChunks;
    cp_async16(dst + k * kRow + 2 * c, src + static_cast<uint64_t>(s_map[k]) * kRow + 2 * c);
  }
  cp_async_commit();
}

// Shared-memory layout of k_planes_admit (in u64 units for the tiles):
//   tile buffer [K * AW * 32] u64, s_map[K] (gather), then the
//   staged class lists when they fit:
//   qc[n_qc] (uint2 program ranges), qc_off[QG + 1] (u32), prog[n_prog] (u16).
struct AdmitSmem {
  size_t tiles, map, lists, total;
};
__host__ __device__ inline AdmitSmem admit_smem_layout(uint32_t K, uint32_t AW, bool gather, size_t list_bytes) {
  AdmitSmem l{};
  l.tiles = 0;
  size_t off = static_cast<size_t>(K) * AW * 32 * 8;
  l.map = off;
  off += gather ? 4ull * K : 0;
  off = (off + 15) & ~static_cast<size_t>(15);
  l.lists = off;
  off += list_bytes;
  l.total = off;
  return l;
}

template <int AW, bool GATHER>
__global__ void __launch_bounds__(kAdmitWarps * 32) k_planes_admit(
    uint32_t G, const uint32_t* __restrict__ goff, const uint8_t* __restrict__ lab, const uint64_t* __restrict__ sig_all,
    uint64_t N, uint32_t R, uint32_t K, uint32_t nlab, const uint32_t* __restrict__ spec, const uint32_t* __restrict__ r_begin,
    int prof, uint32_t base, const uint64_t* __restrict__ rplanes, uint32_t rrows, const uint32_t* __restrict__ row_map,
    uint32_t QG,
    const uint16_t* __restrict__ g_prog, const uint32_t* __restrict__ g_qc_off,
    const uint2* __restrict__ g_qc, uint32_t n_qc, uint32_t n_prog, int stage_lists,
    const uint32_t* __restrict__ row_of, uint32_t out_rows, int accumulate, uint64_t* __restrict__ planes,
    uint32_t* __restrict__ admit, uint32_t* __restrict__ counts) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint32_t tile_cnt[32];
  constexpr uint32_t kRow = AW * 32u;
  const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint32_t GW = (G + 31u) / 32u;
  const uint32_t words = K * AW;
  const size_t list_bytes = stage_lists ? 8ull * n_qc + 4ull * (QG + 1) + 2ull * n_prog : 0;
  const AdmitSmem L = admit_smem_layout(K, AW, GATHER, list_bytes);
  uint64_t* tiles = reinterpret_cast<uint64_t*>(smem_raw);
  uint32_t* s_map = reinterpret_cast<uint32_t*>(smem_raw + L.map);
  // per-batch constants: the row map and (when they fit) the class lists
  const uint32_t* qc_off = g_qc_off;
  const uint2* qc = g_qc;
  const uint16_t* prog = g_prog;
  if (GATHER)
    for (uint32_t i = threadIdx.x; i < K; i += blockDim.x) s_map[i] = row_map[i];
  if (stage_lists) {
    uint2* p2 = reinterpret_cast<uint2*>(smem_raw + L.lists);
    for (uint32_t i = threadIdx.x; i < n_qc; i += blockDim.x) p2[i] = g_qc[i];
    uint32_t* p = reinterpret_cast<uint32_t*>(p2 + n_qc);
    for (uint32_t i = threadIdx.x; i <= QG; i += blockDim.x) p[i] = g_qc_off[i];
    uint16_t* p16 = reinterpret_cast<uint16_t*>(p + QG + 1);
    for (uint32_t i = threadIdx.x; i < n_prog; i += blockDim.x) p16[i] = g_prog[i];
    qc = p2;
    qc_off = p;
    prog = p16;
  }
  __syncthreads();
  for (uint32_t gw = blockIdx.x; gw < GW; gw += gridDim.x) {
    uint64_t* tile = tiles;
    if (GATHER) {
      // one tile buffer (not two, double-buffered): at 35 KB instead of 70 KB
      // per CTA more CTAs share an SM and hide each other's gathers
      __syncthreads();  // every warp is done with the previous tile
      gather_tile_async<AW>(tile, rplanes, rrows, gw, K, s_map);
      cp_async_wait_all();  // this thread's copies; the barrier below covers the others'
    } else {
      __syncthreads();  // the previous tile is no longer read
      fill_tile<AW, false>(tile, gw, G, goff, lab, sig_all, N, R, K, nlab, spec, r_begin, prof, base, nullptr, 0, nullptr);
    }
    if (threadIdx.x < 32) tile_cnt[threadIdx.x] = 0;
    __syncthreads();
    if (!GATHER) {
      if (!row_of) {  // the batch's planes: this tile's rows, contiguous
        uint4* dst = reinterpret_cast<uint4*>(planes + static_cast<uint64_t>(gw) * words * 32);
        const uint4* src = reinterpret_cast<const uint4*>(tile);
        for (uint32_t i = threadIdx.x; i < words * 16; i += blockDim.x) dst[i] = src[i];
      } else {  // one group of the batch: local row k goes to row row_of[k] of out_rows
        constexpr uint32_t kChunks = AW * 16u;  // 16-byte chunks per row
        uint64_t* dst = planes + static_cast<uint64_t>(gw) * out_rows * kRow;
        for (uint32_t i = threadIdx.x; i < K * kChunks; i += blockDim.x) {
          const uint32_t k = i / kChunks, c = i % kChunks;
          reinterpret_cast<uint4*>(dst + static_cast<uint64_t>(row_of[k]) * kRow)[c] =
              reinterpret_cast<const uint4*>(tile + k * kRow)[c];
        }
      }
    }
    const uint64_t* tl = tile + lane;
    const uint32_t in_tile = G - gw * 32u;
    const uint32_t valid_lanes = in_tile >= 32u ? 0xFFFFFFFFu : ((1u << in_tile) - 1u);
    uint32_t my_cnt = 0;
    for (uint32_t qg = wid; qg < QG; qg += nw) {
      const uint32_t e0 = qc_off[qg], e1 = qc_off[qg + 1];
      uint32_t alive = e1 > e0 ? valid_lanes : 0u;  // an empty list: a query of at most one vertex
      for (uint32_t e = e0; e < e1 && alive; ++e) {
        const uint2 pr = qc[e];  // the class's program: prog[pr.x, pr.y)
        uint64_t m[AW];
#pragma unroll
        for (int w = 0; w < AW; ++w) m[w] = ~0ull;
        bool any = true;
        const uint32_t k1 = pr.y;
        // four planes per step between the warp votes
        uint32_t k = pr.x;
        bool live = true;
        for (; k + 4 <= k1; k += 4) {
          const uint32_t off0 = static_cast<uint32_t>(prog[k]) * kRow, off1 = static_cast<uint32_t>(prog[k + 1]) * kRow;
          const uint32_t off2 = static_cast<uint32_t>(prog[k + 2]) * kRow, off3 = static_cast<uint32_t>(prog[k + 3]) * kRow;
          any = false;
#pragma unroll
          for (int w = 0; w < AW; ++w) {
            m[w] &= (tl[off0 + 32 * w] & tl[off1 + 32 * w]) & (tl[off2 + 32 * w] & tl[off3 + 32 * w]);
            any |= m[w] != 0;
          }
          if (!__any_sync(0xFFFFFFFFu, any)) {
            live = false;
            break;
          }
        }
        if (live && k < k1) {
          any = false;
          for (; k < k1; ++k) {
            const uint32_t off = static_cast<uint32_t>(prog[k]) * kRow;
#pragma unroll
            for (int w = 0; w < AW; ++w) m[w] &= tl[off + 32 * w];
          }
#pragma unroll
          for (int w = 0; w < AW; ++w) any |= m[w] != 0;
        }
        const uint32_t word = __ballot_sync(0xFFFFFFFFu, any);
        alive &= word;
      }
      if (lane == 0) admit[static_cast<uint64_t>(qg) * GW + gw] = alive;
      my_cnt += (alive >> lane) & 1u;
    }
    atomicAdd(&tile_cnt[lane], my_cnt);
    __syncthreads();
    if (threadIdx.x < 32 && gw * 32u + threadIdx.x < G) {
      if (accumulate) atomicAdd(&counts[gw * 32u + threadIdx.x], tile_cnt[threadIdx.x]);
      else counts[gw * 32u + threadIdx.x] = tile_cnt[threadIdx.x];
    }
  }
  if (GATHER) cp_async_wait_all();
}

// Planes of a fixed spec for every graph, into out[tile][out_rows][AW][32]
// (rows K .. out_rows - 1 zeroed): the resident planes of the serving loop.
template <int AW>
__global__ void __launch_bounds__(kAdmitWarps * 32) k_build_planes(
    uint32_t G, const uint32_t* __restrict__ goff, const uint8_t* __restrict__ lab, const uint64_t* __restrict__ sig_all,
    uint64_t N, uint32_t R, uint32_t K, uint32_t nlab, const uint32_t* __restrict__ spec, const uint32_t* __restrict__ r_begin,
    int prof, uint32_t base, uint32_t out_rows, uint64_t* __restrict__ out) {
  extern __shared__ uint64_t tile[];  // [K * AW][32]
  const uint32_t GW = (G + 31u) / 32u;
  for (uint32_t gw = blockIdx.x; gw < GW; gw += gridDim.x) {
    __syncthreads();
    fill_tile<AW, false>(tile, gw, G, goff, lab, sig_all, N, R, K, nlab, spec, r_begin, prof, base, nullptr, 0, nullptr);
    __syncthreads();
    uint4* dst = reinterpret_cast<uint4*>(out + static_cast<uint64_t>(gw) * out_rows * AW * 32);
    const uint4* src = reinterpret_cast<const uint4*>(tile);
    const uint32_t have = K * AW * 16, all = out_rows * AW * 16;
    for (uint32_t i = threadIdx.x; i < all; i += blockDim.x) dst[i] = i < have ? src[i] : make_uint4(0, 0, 0, 0);
  }
}

// Largest count of label l at iteration r over all vertices: cmax[r * 16 + l].
__global__ void k_sig_cmax(const uint64_t* __restrict__ sig_all, uint64_t N, uint32_t R, unsigned int* __restrict__ cmax) {
  for (uint32_t r = 0; r < R; ++r) {
    uint32_t mx[16];
#pragma unroll
    for (int l = 0; l < 16; ++l) mx[l] = 0;
    for (uint64_t v = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; v < N;
         v += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
      const uint64_t sv = sig_all[static_cast<uint64_t>(r) * N + v];
#pragma unroll
      for (int l = 0; l < 16; ++l) mx[l] = max(mx[l], static_cast<uint32_t>((sv >> (4 * l)) & 0xFull));
    }
#pragma unroll
    for (int l = 0; l < 16; ++l) {
      const uint32_t m = __reduce_max_sync(0xFFFFFFFFu, mx[l]);
      if ((threadIdx.x & 31u) == 0 && m) atomicMax(&cmax[r * 16 + l], m);
    }
  }
}

// Vertices per label value (shared-memory bins, one atomic per bin per block).
__global__ void k_label_hist(const uint8_t* __restrict__ lab, uint64_t n, unsigned long long* __restrict__ hist) {
  __shared__ unsigned int bins[256];
  for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) bins[i] = 0;
  __syncthreads();
  for (uint64_t v = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; v < n;
       v += static_cast<uint64_t>(gridDim.x) * blockDim.x)
    atomicAdd(&bins[lab[v]], 1u);
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x)
    if (bins[i]) atomicAdd(&hist[i], static_cast<unsigned long long>(bins[i]));
}

}  // namespace

int ensure_label_hist(Queue* q, Graph* g) {
  if (g->label_hist.size() == 256) return SIGMO_OK;
  void* buf = nullptr;
  SIGMO_TRY(tmp_alloc(q, &buf, 256 * 8));
  int rc = SIGMO_OK;
  if (cudaMemsetAsync(buf, 0, 256 * 8, q->stream) != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "memset failed");
  if (!rc && g->total_nodes) {
    k_label_hist<<<grid_for(g->total_nodes, 256, 148u * 4u), 256, 0, q->stream>>>(g->node_labels, g->total_nodes,
                                                                                 static_cast<unsigned long long*>(buf));
    rc = check_launch(q, "k_label_hist");
  }
  std::vector<uint64_t> h(256, 0);
  if (!rc && (cudaMemcpyAsync(h.data(), buf, 256 * 8, cudaMemcpyDeviceToHost, q->stream) != cudaSuccess ||
              cudaStreamSynchronize(q->stream) != cudaSuccess))
    rc = fail(SIGMO_ERR_CUDA, "label histogram read-back failed");
  dev_free(q, buf);
  if (!rc) g->label_hist = std::move(h);
  return rc;
}

size_t planes_admit_smem(uint32_t K, uint32_t AW) {
  return admit_smem_layout(K, AW, false, 0).total;
}

namespace {

// What one admission launch needs of a program: the whole batch's, or one
// group's (local ids; planes scattered to row_of).
struct AdmitView {
  uint32_t K, nlab, QG;
  const uint32_t *spec, *r_begin;
  const uint32_t* qc_off;  // [QG + 1] entries of qc per query graph
  const uint32_t* qc;      // per entry, its class's program range in prog (u32 pairs)
  const uint32_t* row_of;  // group launches: local plane row -> row of the batch's plane array
  const uint16_t* prog;
  size_t n_qc, n_prog;
  uint32_t out_rows;
  int accumulate;
};

template <int AW, bool GATHER>
int admit_launch(Queue* q, const Graph* data, const uint64_t* sig_all, uint32_t R, const AdmitView& v, const uint64_t* rplanes,
                 uint32_t rrows, const uint32_t* row_map, uint64_t* planes, uint32_t* admit, uint32_t* counts) {
  const uint32_t G = data->num_graphs, GW = (G + 31u) / 32u, QG = v.QG;
  const uint32_t n_qc = static_cast<uint32_t>(v.n_qc), n_prog = static_cast<uint32_t>(v.n_prog);
  const size_t list_bytes = 8ull * n_qc + 4ull * (QG + 1) + 2ull * n_prog;
  const size_t base = admit_smem_layout(v.K, AW, GATHER, 0).total;
  // stage the class lists when the block still fits three to an SM
  const int stage = base + list_bytes <= 72u * 1024u ? 1 : 0;
  const size_t smem = admit_smem_layout(v.K, AW, GATHER, stage ? list_bytes : 0).total;
  if (smem > 220u * 1024u) return fail(SIGMO_ERR_DOMAIN, "k_planes_admit needs %zu bytes of shared memory", smem);
  const unsigned block = 32u * kAdmitWarps;
  int per_sm = 0, sms = 0;
  SIGMO_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, q->device));
  SIGMO_TRY(allow_max_dynamic_smem(reinterpret_cast<const void*>(k_planes_admit<AW, GATHER>), q->device));
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_planes_admit<AW, GATHER>, block, smem);
  if (e != cudaSuccess) return fail(SIGMO_ERR_CUDA, "k_planes_admit shared-memory setup failed: %s", cudaGetErrorString(e));
  const uint64_t grid = std::min<uint64_t>(GW, static_cast<uint64_t>(std::max(per_sm, 1)) * sms);
  k_planes_admit<AW, GATHER><<<grid, block, smem, q->stream>>>(
      G, data->graph_offsets, data->node_labels, sig_all, data->total_nodes, R, v.K, v.nlab, v.spec, v.r_begin, q->opts.profile,
      data->vertex_base, rplanes, rrows, row_map, QG, v.prog, v.qc_off, reinterpret_cast<const uint2*>(v.qc), n_qc,
      n_prog, stage,
      v.row_of, v.out_rows, v.accumulate, planes, admit, counts);
  return check_launch(q, "k_planes_admit");
}

AdmitView whole_batch(const Graph* query, const PlaneProgram& pp) {
  return AdmitView{pp.K, pp.nlab, query->num_graphs, pp.spec, pp.r_begin, pp.qc_off, pp.qc, nullptr, pp.prog, pp.h_qc_n,
                   pp.h_prog.size(), pp.K, 0};
}

}  // namespace

int launch_planes_admit(Queue* q, const Graph* query, const Graph* data, const uint64_t* sig_all, uint32_t R,
                        const PlaneProgram& pp, uint64_t* planes, uint32_t* admit, uint32_t* counts) {
  if (!data->num_graphs) return SIGMO_OK;
  const AdmitView v = whole_batch(query, pp);
  switch (data->adj_words) {
    case 1: return admit_launch<1, false>(q, data, sig_all, R, v, nullptr, 0, nullptr, planes, admit, counts);
    case 2: return admit_launch<2, false>(q, data, sig_all, R, v, nullptr, 0, nullptr, planes, admit, counts);
    default: return admit_launch<4, false>(q, data, sig_all, R, v, nullptr, 0, nullptr, planes, admit, counts);
  }
}

int launch_planes_admit_group(Queue* q, const Graph* query, const Graph* data, const uint64_t* sig_all, uint32_t R,
                              const PlaneGroup& grp, uint32_t K_total, uint64_t* planes, uint32_t* admit, uint32_t* counts) {
  if (!data->num_graphs || grp.q1 <= grp.q0) return SIGMO_OK;
  const uint32_t GW = (data->num_graphs + 31u) / 32u;
  const AdmitView v{grp.K,      grp.nlab, grp.q1 - grp.q0, grp.spec, grp.r_begin, grp.qc_off, grp.qc, grp.row_of, grp.prog,
                    grp.n_qc, grp.n_prog, K_total, 1};
  uint32_t* adm = admit + static_cast<uint64_t>(grp.q0) * GW;
  switch (data->adj_words) {
    case 1: return admit_launch<1, false>(q, data, sig_all, R, v, nullptr, 0, nullptr, planes, adm, counts);
    case 2: return admit_launch<2, false>(q, data, sig_all, R, v, nullptr, 0, nullptr, planes, adm, counts);
    default: return admit_launch<4, false>(q, data, sig_all, R, v, nullptr, 0, nullptr, planes, adm, counts);
  }
}

int launch_planes_admit_resident(Queue* q, const Graph* query, const Graph* data, const ResidentPlanes& rp,
                                 const PlaneProgram& pp, const uint32_t* row_map, uint32_t* admit, uint32_t* counts) {
  if (!data->num_graphs) return SIGMO_OK;
  const AdmitView v = whole_batch(query, pp);
  switch (data->adj_words) {
    case 1: return admit_launch<1, true>(q, data, nullptr, 0, v, rp.planes, rp.rows, row_map, nullptr, admit, counts);
    case 2: return admit_launch<2, true>(q, data, nullptr, 0, v, rp.planes, rp.rows, row_map, nullptr, admit, counts);
    default: return admit_launch<4, true>(q, data, nullptr, 0, v, rp.planes, rp.rows, row_map, nullptr, admit, counts);
  }
}

// Resident planes of every (label) and (iteration, label, count) that occurs
// in the database: label planes for each label present and the wildcard,
// thresholds c = 1..cmax(r, l), then one zero row.
int build_resident_planes(Queue* q, Graph* data, const uint64_t* sig_all, uint32_t R, ResidentPlanes* out) {
  SIGMO_TRY(ensure_label_hist(q, data));
  const uint64_t N = data->total_nodes;
  const uint32_t G = data->num_graphs, GW = (G + 31u) / 32u, AW = data->adj_words;
  std::vector<unsigned int> cmax(16ull * (R ? R : 1), 0);
  if (R && N) {
    void* d = nullptr;
    SIGMO_TRY(dev_alloc(q, &d, 4ull * 16 * R));
    int rc = cudaMemsetAsync(d, 0, 4ull * 16 * R, q->stream) == cudaSuccess ? SIGMO_OK : fail(SIGMO_ERR_CUDA, "memset failed");
    if (!rc) {
      k_sig_cmax<<<grid_for(N, 256, 148u * 8u), 256, 0, q->stream>>>(sig_all, N, R, static_cast<unsigned int*>(d));
      rc = check_launch(q, "k_sig_cmax");
    }
    if (!rc && (cudaMemcpyAsync(cmax.data(), d, 4ull * 16 * R, cudaMemcpyDeviceToHost, q->stream) != cudaSuccess ||
                cudaStreamSynchronize(q->stream) != cudaSuccess))
      rc = fail(SIGMO_ERR_CUDA, "cmax read-back failed");
    dev_free(q, d);
    SIGMO_TRY(rc);
  }
  std::vector<uint32_t> spec;
  out->label_row.assign(256, 0);
  for (uint32_t l = 0; l < 256; ++l)
    if (data->label_hist[l] || l == kWildcard) {
      out->label_row[l] = static_cast<uint32_t>(spec.size());
      spec.push_back(0x80000000u | l);
    }
  const uint32_t nlab = static_cast<uint32_t>(spec.size());
  std::vector<uint32_t> r_begin(R + 1, 0);
  out->base_row.assign(16ull * R, 0);
  out->cmax.assign(16ull * R, 0);
  for (uint32_t r = 0; r < R; ++r) {
    r_begin[r] = static_cast<uint32_t>(spec.size());
    for (uint32_t l = 0; l < 16; ++l) {
      const uint32_t cm = cmax[r * 16 + l];
      out->cmax[r * 16 + l] = static_cast<uint8_t>(cm);
      out->base_row[r * 16 + l] = static_cast<uint32_t>(spec.size());
      for (uint32_t c = 1; c <= cm; ++c) spec.push_back((r << 16) | (l << 8) | c);
    }
  }
  r_begin[R] = static_cast<uint32_t>(spec.size());
  const uint32_t K = static_cast<uint32_t>(spec.size());
  out->zero_row = K;
  for (uint32_t l = 0; l < 256; ++l)
    if (!data->label_hist[l] && l != kWildcard) out->label_row[l] = K;
  out->rows = K + 1;
  out->R = R;
  const size_t smem = static_cast<size_t>(K) * AW * 32 * 8;
  if (smem > 200u * 1024u) return fail(SIGMO_ERR_DOMAIN, "the database needs %u resident planes (too many for one tile)", K);
  void* dspec = nullptr;
  void* drb = nullptr;
  SIGMO_TRY(dev_alloc(q, &dspec, 4ull * K));
  SIGMO_TRY(dev_alloc(q, &drb, 4ull * (R + 1)));
  int rc = SIGMO_OK;
  if (cudaMemcpyAsync(dspec, spec.data(), 4ull * K, cudaMemcpyHostToDevice, q->stream) != cudaSuccess ||
      cudaMemcpyAsync(drb, r_begin.data(), 4ull * (R + 1), cudaMemcpyHostToDevice, q->stream) != cudaSuccess)
    rc = fail(SIGMO_ERR_CUDA, "H2D copy failed");
  if (!rc) rc = dev_alloc(q, reinterpret_cast<void**>(&out->planes), 8ull * GW * out->rows * AW * 32 + 8);
  if (!rc && GW) {
    int per_sm = 0, sms = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, q->device);
    const unsigned block = 32u * kAdmitWarps;
#define SIGMO_BUILD(AWV)                                                                                             \
  if (e == cudaSuccess &&                                                                                             \
      allow_max_dynamic_smem(reinterpret_cast<const void*>(k_build_planes<AWV>), q->device) != SIGMO_OK)               \
    e = cudaErrorInvalidValue;                                                                                         \
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_build_planes<AWV>, block, smem);  \
  if (e == cudaSuccess)                                                                                              \
    k_build_planes<AWV><<<std::min<uint64_t>(GW, static_cast<uint64_t>(std::max(per_sm, 1)) * sms), block, smem,      \
                          q->stream>>>(G, data->graph_offsets, data->node_labels, sig_all, N, R, K, nlab,            \
                                       static_cast<const uint32_t*>(dspec), static_cast<const uint32_t*>(drb),        \
                                       q->opts.profile, data->vertex_base, out->rows, out->planes)
    switch (AW) {
      case 1: SIGMO_BUILD(1); break;
      case 2: SIGMO_BUILD(2); break;
      default: SIGMO_BUILD(4); break;
    }
#undef SIGMO_BUILD
    if (e != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "k_build_planes setup failed: %s", cudaGetErrorString(e));
    if (!rc) rc = check_launch(q, "k_build_planes");
  }
  if (!rc && cudaStreamSynchronize(q->stream) != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "resident plane build failed");
  dev_free(q, dspec);
  dev_free(q, drb);
  return rc;
}

}  // namespace sigmo_b200
