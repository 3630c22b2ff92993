// GMCR: the query-graph -> data-graph mapping (isomorphism::mapping::GMCR,
// library/include/gmcr.hpp:33-128).  A pair (query graph q, data graph g) is
// admitted when every vertex of q has at least one range-masked candidate in
// g (getCandidatesCount(q_i, start_g, end_g) > 0, candidates.hpp:86-104).
//
// Instead of evaluating the predicate per pair twice with a serial scan in
// between, the mapping is built from one streaming pass over the bitset:
//   1. NE[j][g/32]: bit g = query vertex j has a candidate in data graph g
//      (one read of the bitset; lane = data graph, ballot per 32 graphs);
//   2. admit[q][g/32] = AND of NE over q's vertices, and per-graph counts;
//   3. a device scan of the counts (the segment offsets);
//   4. the fill, writing each segment's query ids in ascending order.
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <mutex>

#include "internal.hpp"

namespace sigmo_b200 {
namespace {

constexpr unsigned kNeRowsPerBlock = 64;
constexpr unsigned kNeBatch = 8;  // rows whose words are loaded together

// Lane = data graph, warp = 32 consecutive graphs (their words are
// contiguous, so a warp's loads for one row cover ~35 consecutive words).
// kNeBatch rows are read per pass over the graph's words so that many loads
// are in flight per lane.
__global__ void k_gmcr_ne(const uint32_t* __restrict__ bits, uint64_t Wp, uint64_t Qn, const uint32_t* __restrict__ dgoff,
                          uint32_t G, uint32_t GW, int prof, uint32_t* __restrict__ NE) {
  const unsigned lane = threadIdx.x & 31u;
  const uint32_t gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (gw >= GW) return;
  const uint32_t g = gw * 32u + lane;
  uint32_t s = 0, e = 0, i0 = 0, i1 = 0;
  if (g < G) {
    s = dgoff[g];
    e = dgoff[g + 1];
    if (e > s) {
      i0 = s >> 5;
      i1 = (e + 31u) >> 5;
    }
  }
  const uint64_t j0 = static_cast<uint64_t>(blockIdx.y) * kNeRowsPerBlock;
  const uint64_t j1 = j0 + kNeRowsPerBlock < Qn ? j0 + kNeRowsPerBlock : Qn;
  // The range masks of this graph's words are the same for every row: a graph
  // of <= 65 vertices spans at most kNeWords words, whose masks are computed
  // once (a zero mask, REF_PTX's dropped last word, is not even loaded).
  constexpr uint32_t kNeWords = 3;
  const bool few = i1 - i0 <= kNeWords;
  uint32_t mk[kNeWords];
#pragma unroll
  for (uint32_t w = 0; w < kNeWords; ++w) mk[w] = few && i0 + w < i1 ? range_mask(i0 + w, s, e, prof) : 0u;
  for (uint64_t j = j0; j < j1; j += kNeBatch) {
    uint32_t acc[kNeBatch];
#pragma unroll
    for (uint32_t k = 0; k < kNeBatch; ++k) acc[k] = 0;
    if (few) {
#pragma unroll
      for (uint32_t w = 0; w < kNeWords; ++w) {
        if (!mk[w]) continue;
        const uint32_t* col = bits + j * Wp + i0 + w;
#pragma unroll
        for (uint32_t k = 0; k < kNeBatch; ++k)
          if (j + k < j1) acc[k] |= col[k * Wp] & mk[w];
      }
    } else {
      for (uint32_t i = i0; i < i1; ++i) {
        const uint32_t m = range_mask(i, s, e, prof);
        const uint32_t* col = bits + j * Wp + i;
#pragma unroll
        for (uint32_t k = 0; k < kNeBatch; ++k)
          if (j + k < j1) acc[k] |= col[k * Wp] & m;
      }
    }
#pragma unroll
    for (uint32_t k = 0; k < kNeBatch; ++k) {
      const uint32_t word = __ballot_sync(0xFFFFFFFFu, acc[k] != 0);
      if (lane == 0 && j + k < j1) NE[(j + k) * GW + gw] = word;
    }
  }
}

// Warp per 32 data graphs; lanes take query graphs 32 at a time.
// NE rows are indexed by query vertex, or by the vertex's class when cls is
// given (the batched form stores one row per class of identical vertices).
__global__ void k_gmcr_admit(const uint32_t* __restrict__ NE, uint32_t GW, const uint32_t* __restrict__ qgoff, uint32_t QG,
                             uint32_t G, const uint32_t* __restrict__ cls, uint32_t* __restrict__ admit,
                             uint32_t* __restrict__ counts) {
  const unsigned lane = threadIdx.x & 31u;
  const uint32_t warp = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t gw = warp; gw < GW; gw += nwarps) {
    const uint32_t valid = (G - gw * 32u) >= 32u ? 0xFFFFFFFFu : ((1u << (G - gw * 32u)) - 1u);
    uint32_t cnt = 0;
    for (uint32_t q0 = 0; q0 < QG; q0 += 32) {
      const uint32_t q = q0 + lane;
      uint32_t a = 0;
      if (q < QG) {
        const uint32_t off = qgoff[q], n = qgoff[q + 1] - off;
        if (n > 1) {
          a = valid;
          for (uint32_t j = 0; j < n && a; ++j) {
            const uint32_t row = cls ? cls[off + j] : off + j;
            a &= NE[static_cast<uint64_t>(row) * GW + gw];
          }
        }
        admit[static_cast<uint64_t>(q) * GW + gw] = a;
      }
#pragma unroll 8
      for (unsigned b = 0; b < 32; ++b) {
        const uint32_t c = __popc(__ballot_sync(0xFFFFFFFFu, (a >> b) & 1u));
        if (lane == b) cnt += c;
      }
    }
    const uint32_t g = gw * 32u + lane;
    if (g < G) counts[g] = cnt;
  }
}

// Segment fill: lane = data graph; query ids visited in ascending order, so
// every segment is sorted.
__global__ void k_gmcr_fill(const uint32_t* __restrict__ admit, uint32_t GW, uint32_t QG, uint32_t G,
                            const uint32_t* __restrict__ offsets, uint32_t* __restrict__ indices,
                            uint32_t* __restrict__ pair_graph, uint64_t capacity) {
  const unsigned lane = threadIdx.x & 31u;
  const uint32_t warp = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t gw = warp; gw < GW; gw += nwarps) {
    const uint32_t g = gw * 32u + lane;
    uint64_t cur = g < G ? offsets[g] : 0;
    uint32_t q = 0;
    for (; q + 8 <= QG; q += 8) {  // eight admission words in flight
      uint32_t a[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) a[k] = admit[static_cast<uint64_t>(q + k) * GW + gw];
#pragma unroll
      for (int k = 0; k < 8; ++k)
        if ((a[k] >> lane) & 1u) {
          if (cur < capacity) {
            indices[cur] = q + k;
            if (pair_graph) pair_graph[cur] = g;
          }
          ++cur;
        }
    }
    for (; q < QG; ++q) {
      const uint32_t a = admit[static_cast<uint64_t>(q) * GW + gw];
      if ((a >> lane) & 1u) {
        if (cur < capacity) {
          indices[cur] = q;
          if (pair_graph) pair_graph[cur] = g;
        }
        ++cur;
      }
    }
  }
}

}  // namespace

// Admission, counts, scan and fill from an NE matrix (rows per query vertex,
// or per class when cls != nullptr).  With sync_total the total is read back
// and the index arrays sized exactly (the reference reads it back too,
// gmcr.hpp:80); otherwise capacity_hint bounds them.
int launch_gmcr_from_admit(Queue* q, const Graph* query, const Graph* data, const uint32_t* admit, const uint32_t* counts,
                           Gmcr* m, bool sync_total, uint64_t capacity_hint) {
  const uint32_t G = data->num_graphs, QG = query->num_graphs;
  const uint32_t GW = (G + 31u) / 32u;
  if (m->offsets && m->num_data_graphs != G) {
    dev_free(q, m->offsets);
    m->offsets = nullptr;
  }
  if (!m->offsets) SIGMO_TRY(dev_alloc(q, reinterpret_cast<void**>(&m->offsets), sizeof(uint32_t) * (G + 1ull)));
  m->num_data_graphs = G;
  m->counts_valid = false;
  SIGMO_CUDA_TRY(cudaMemsetAsync(m->offsets, 0, sizeof(uint32_t) * (G + 1ull), q->stream));
  size_t cub_bytes = 0;
  if (G) cub::DeviceScan::InclusiveSum(nullptr, cub_bytes, static_cast<uint32_t*>(nullptr), static_cast<uint32_t*>(nullptr),
                                       static_cast<int>(G), q->stream);
  void* cub_tmp = nullptr;
  SIGMO_TRY(tmp_alloc(q, &cub_tmp, cub_bytes + 256));
  int rc = SIGMO_OK;
  if (G && QG) {
    cudaError_t e = cub::DeviceScan::InclusiveSum(cub_tmp, cub_bytes, counts, m->offsets + 1, static_cast<int>(G), q->stream);
    if (e != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "device scan failed: %s", cudaGetErrorString(e));
    q->launches += 2;
  }
  uint64_t cap = capacity_hint;
  if (!rc && sync_total) {
    uint32_t* pinned = static_cast<uint32_t*>(q->pinned);
    cudaError_t e = cudaMemcpyAsync(pinned, m->offsets + G, sizeof(uint32_t), cudaMemcpyDeviceToHost, q->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(q->stream);
    if (e != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "reading the GMCR total failed: %s", cudaGetErrorString(e));
    m->total = *pinned;
    cap = m->total;
  }
  if (!rc && (cap > m->capacity || !m->indices)) {
    dev_free(q, m->indices);
    dev_free(q, m->pair_graph);
    dev_free(q, m->counts);
    m->indices = m->pair_graph = nullptr;
    m->counts = nullptr;
    // grow by half again at least, so a sequence of growing batches
    // reallocates O(log) times
    const uint64_t n = std::max<uint64_t>(cap ? cap : 1, m->capacity + m->capacity / 2);
    m->capacity = 0;
    rc = dev_alloc(q, reinterpret_cast<void**>(&m->indices), sizeof(uint32_t) * n);
    if (!rc) rc = dev_alloc(q, reinterpret_cast<void**>(&m->pair_graph), sizeof(uint32_t) * n);
    if (!rc) rc = dev_alloc(q, reinterpret_cast<void**>(&m->counts), sizeof(uint64_t) * n);
    if (!rc) m->capacity = n;
  }
  if (!rc && G && QG) {
    k_gmcr_fill<<<grid_for(GW * 32ull, 256, 148u * 16u), 256, 0, q->stream>>>(admit, GW, QG, G, m->offsets, m->indices,
                                                                                m->pair_graph, m->capacity);
    rc = check_launch(q, "k_gmcr_fill");
  }
  dev_free(q, cub_tmp);
  return rc;
}

// Admission and counts from an NE matrix (rows per query vertex, or per class
// when cls != nullptr), then launch_gmcr_from_admit.
int launch_gmcr_from_ne(Queue* q, const Graph* query, const Graph* data, const uint32_t* NE, const uint32_t* cls, Gmcr* m,
                        bool sync_total, uint64_t capacity_hint) {
  const uint32_t G = data->num_graphs, QG = query->num_graphs;
  const uint32_t GW = (G + 31u) / 32u;
  const uint64_t admit_words = static_cast<uint64_t>(QG) * GW;
  auto al = [](size_t x) { return (x + 255) & ~static_cast<size_t>(255); };
  void* buf = nullptr;
  SIGMO_TRY(tmp_alloc(q, &buf, al(admit_words * 4) + al(G * 4ull) + 256));
  uint32_t* admit = static_cast<uint32_t*>(buf);
  uint32_t* counts = reinterpret_cast<uint32_t*>(static_cast<char*>(buf) + al(admit_words * 4));
  int rc = SIGMO_OK;
  if (G && QG) {
    k_gmcr_admit<<<grid_for(GW * 32ull, 256, 148u * 16u), 256, 0, q->stream>>>(NE, GW, query->graph_offsets, QG, G, cls, admit, counts);
    rc = check_launch(q, "k_gmcr_admit");
  }
  if (!rc) rc = launch_gmcr_from_admit(q, query, data, admit, counts, m, sync_total, capacity_hint);
  dev_free(q, buf);
  return rc;
}

// GMCR from the candidate bitset: NE per query vertex, then the above.
int launch_gmcr(Queue* q, const Graph* query, const Graph* data, const Candidates* c, Gmcr* m, bool sync_total,
                uint64_t capacity_hint) {
  const uint32_t G = data->num_graphs;
  const uint32_t GW = (G + 31u) / 32u;
  const uint64_t Qn = query->total_nodes;
  void* ne = nullptr;
  SIGMO_TRY(tmp_alloc(q, &ne, 4ull * Qn * GW + 4));
  uint32_t* NE = static_cast<uint32_t*>(ne);
  int rc = SIGMO_OK;
  if (G && query->num_graphs && Qn) {
    dim3 grid_ne((GW + 7u) / 8u, static_cast<unsigned>((Qn + kNeRowsPerBlock - 1) / kNeRowsPerBlock));
    if (grid_ne.y > 65535u) rc = fail(SIGMO_ERR_DOMAIN, "too many query vertices (%llu)", (unsigned long long)Qn);
    if (!rc) {
      k_gmcr_ne<<<grid_ne, 256, 0, q->stream>>>(c->bits, c->Wp, Qn, data->graph_offsets, G, GW, q->opts.profile, NE);
      rc = check_launch(q, "k_gmcr_ne");
    }
  }
  if (!rc) rc = launch_gmcr_from_ne(q, query, data, NE, nullptr, m, sync_total, capacity_hint);
  dev_free(q, ne);
  return rc;
}

// ---- GMCR without device allocation ----------------------------------------
// Some callers cannot allocate device memory while this step runs: code that
// works inside a fixed device-memory arena owned by another allocator (a host
// framework's caching allocator that has reserved the free memory), real-time
// services that forbid cudaMalloc/cudaFree on their request path after
// start-up, and callers that cannot afford the implicit synchronisation an
// allocation or free may bring.  sigmo_gmcr_generate_noalloc computes the same
// GMCR as sigmo_gmcr_generate with every intermediate (non-empty matrix,
// admission words, per-graph counts, scan temporary storage) in one
// file-scope device array and the results in buffers the caller owns.

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB; every GPU that loads the library holds it until exit
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_addr[128] = {};  // device address of g_noalloc_scratch on each device

// Device address of the scratch array on `device`, which must be current.
// In host code the array's name is only a host-side stand-in, so the address
// is resolved once per device with cudaGetSymbolAddress (the first call on a
// device does this set-up).
int noalloc_scratch(int device, void** out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (device < 0 || device >= 128) return fail(SIGMO_ERR_NO_DEVICE, "device %d out of range", device);
  if (!g_noalloc_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(SIGMO_ERR_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch) failed: %s", cudaGetErrorString(e));
    g_noalloc_addr[device] = p;
  }
  *out = g_noalloc_addr[device];
  return SIGMO_OK;
}

}  // namespace
}  // namespace sigmo_b200

extern "C" int sigmo_gmcr_generate_noalloc(sigmo_queue_t q, sigmo_graph_t query, sigmo_graph_t data, sigmo_candidates_t c,
                                           uint32_t* d_offsets, uint32_t* d_indices, uint64_t capacity, uint64_t* total) {
  using namespace sigmo_b200;
  if (!q || !query || !data || !c || !d_offsets || !total || (!d_indices && capacity))
    return fail(SIGMO_ERR_INVALID, "sigmo_gmcr_generate_noalloc: null argument");
  if (c->rows != query->total_nodes || c->targets != data->total_nodes)
    return fail(SIGMO_ERR_INVALID, "candidate bitset does not match the graphs");
  SIGMO_CUDA_TRY(cudaSetDevice(q->device));
  const uint32_t G = data->num_graphs, QG = query->num_graphs, GW = (G + 31u) / 32u;
  const uint64_t Qn = query->total_nodes;
  size_t cub_bytes = 0;
  if (G)
    SIGMO_CUDA_TRY(cub::DeviceScan::InclusiveSum(nullptr, cub_bytes, static_cast<uint32_t*>(nullptr),
                                                 static_cast<uint32_t*>(nullptr), static_cast<int>(G), q->stream));
  auto al = [](size_t x) { return (x + 255) & ~static_cast<size_t>(255); };
  const size_t need = al(4ull * Qn * GW) + al(4ull * QG * GW) + al(4ull * G) + al(cub_bytes);
  if (need > kNoAllocScratchBytes)
    return fail(SIGMO_ERR_DOMAIN,
                "sigmo_gmcr_generate_noalloc: %zu bytes of scratch needed (%llu query vertices x %u data graphs), the "
                "static scratch holds %zu; use sigmo_gmcr_generate",
                need, static_cast<unsigned long long>(Qn), G, kNoAllocScratchBytes);
  void* scratch = nullptr;
  SIGMO_TRY(noalloc_scratch(q->device, &scratch));
  char* p = static_cast<char*>(scratch);
  uint32_t* NE = reinterpret_cast<uint32_t*>(p);
  p += al(4ull * Qn * GW);
  uint32_t* admit = reinterpret_cast<uint32_t*>(p);
  p += al(4ull * QG * GW);
  uint32_t* counts = reinterpret_cast<uint32_t*>(p);
  p += al(4ull * G);
  void* cub_tmp = p;
  // d_offsets[0] must start at zero; NE, admit and counts are fully written below.
  SIGMO_CUDA_TRY(cudaMemsetAsync(d_offsets, 0, sizeof(uint32_t) * (G + 1ull), q->stream));
  if (G && QG && Qn) {
    dim3 grid_ne((GW + 7u) / 8u, static_cast<unsigned>((Qn + kNeRowsPerBlock - 1) / kNeRowsPerBlock));
    if (grid_ne.y > 65535u) return fail(SIGMO_ERR_DOMAIN, "too many query vertices (%llu)", static_cast<unsigned long long>(Qn));
    k_gmcr_ne<<<grid_ne, 256, 0, q->stream>>>(c->bits, c->Wp, Qn, data->graph_offsets, G, GW, q->opts.profile, NE);
    SIGMO_TRY(check_launch(q, "k_gmcr_ne"));
    k_gmcr_admit<<<grid_for(GW * 32ull, 256, 148u * 16u), 256, 0, q->stream>>>(NE, GW, query->graph_offsets, QG, G, nullptr,
                                                                                admit, counts);
    SIGMO_TRY(check_launch(q, "k_gmcr_admit"));
    SIGMO_CUDA_TRY(cub::DeviceScan::InclusiveSum(cub_tmp, cub_bytes, counts, d_offsets + 1, static_cast<int>(G), q->stream));
    q->launches += 2;
  }
  uint32_t* pinned = static_cast<uint32_t*>(q->pinned);
  SIGMO_CUDA_TRY(cudaMemcpyAsync(pinned, d_offsets + G, sizeof(uint32_t), cudaMemcpyDeviceToHost, q->stream));
  SIGMO_CUDA_TRY(cudaStreamSynchronize(q->stream));
  *total = *pinned;
  if (*total > capacity)
    return fail(SIGMO_ERR_INVALID, "sigmo_gmcr_generate_noalloc: %llu admitted pairs exceed the index buffer of %llu entries",
                static_cast<unsigned long long>(*total), static_cast<unsigned long long>(capacity));
  if (G && QG && Qn) {
    k_gmcr_fill<<<grid_for(GW * 32ull, 256, 148u * 16u), 256, 0, q->stream>>>(admit, GW, QG, G, d_offsets, d_indices, nullptr,
                                                                                capacity);
    SIGMO_TRY(check_launch(q, "k_gmcr_fill"));
  }
  return SIGMO_OK;
}
