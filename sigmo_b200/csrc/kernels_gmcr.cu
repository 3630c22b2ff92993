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

#include "bulk.cuh"
#include "internal.hpp"

namespace sigmo_b200 {
namespace {

// Non-empty pass: NE[j][g/32] bit g%32 = query vertex j has a range-masked
// candidate in data graph g.  A CTA owns 256 consecutive data graphs (8 NE
// words, lane = data graph) and a run of kNeRowsPerCta bitset rows.  The
// words its graphs span in a row, [ws, we) rounded out to 16-byte
// boundaries, arrive in shared memory by bulk asynchronous copies (one per
// row, issued by the lanes of warp 0) into a ring of kNeStages stages whose
// completion is counted on one mbarrier per stage; each warp then reads its
// graphs' 1-3 words per row from shared memory, ANDs them with the graph's
// range masks (computed once: only a graph's first and last words are
// partial, candidates.hpp:91-99) and votes the row's NE word.  So DRAM sees
// every bitset byte once in 16-byte-aligned bursts, and the per-row work is a
// few shared-memory loads, logic ops, a vote and a store per warp.  A CTA
// whose span exceeds one stage reads global memory instead (same results).
// Waits are bounded: a thread whose wait runs out reads that chunk from
// global memory, and warp 0 stops refilling a stage whose phase it did not
// see complete (it waits for it again, bounded, before the CTA exits).
constexpr uint32_t kNeThreads = 256;
constexpr uint32_t kNeStages = 2;
constexpr uint32_t kNeStageWords = 6144;  // 24 KiB per stage (4 CTAs per SM)
constexpr uint32_t kNeRowsPerCta = 512;
constexpr uint32_t kNeSleepNs = 20000;  // longest suspension per poll of a stage's mbarrier
constexpr uint32_t kNePolls = 1u << 16;  // polls before a wait gives up (about a second at most)
constexpr uint32_t kNePadWords = 4;       // slack for the fixed three-word reads of the last row
constexpr size_t kNeSmemBytes = sizeof(uint32_t) * (kNeStages * kNeStageWords + kNePadWords);

struct NeLane {
  uint32_t i0, nw;      // the graph's first word and word count (0: empty or past the last graph)
  uint32_t mf, ml;      // range masks of its first and last words
  uint32_t m0, m1, m2;  // masks of words 0..2 (nw <= 3)
  uint32_t o1, o2;      // word offsets of words 1 and 2, clamped to the graph's words
};

// The NE bit of one row for a lane, from the row's words starting at `row`
// (word i0 of the graph at row[0]).
__device__ __forceinline__ bool ne_any_few(const uint32_t* row, const NeLane& L) {
  return ((row[0] & L.m0) | (row[L.o1] & L.m1) | (row[L.o2] & L.m2)) != 0u;
}
__device__ __forceinline__ bool ne_any_wide(const uint32_t* row, const NeLane& L) {
  uint32_t acc = 0;
  for (uint32_t k = 0; k < L.nw; ++k) acc |= row[k] & (k == 0 ? L.mf : (k + 1 == L.nw ? L.ml : 0xFFFFFFFFu));
  return acc != 0u;
}

// Warp 0 of k_gmcr_ne: the bulk copies of chunk c (RS rows of SW words from
// row j0 + c * RS on, word ws on) into stage c % kNeStages.
__device__ __forceinline__ void ne_issue(uint32_t c, uint32_t lane, uint32_t RS, uint32_t SW, uint32_t nrows, uint64_t j0,
                                         uint32_t ws, uint64_t Wp, const uint32_t* __restrict__ bits, uint32_t* s_stage,
                                         uint64_t* s_bar, uint32_t* s_live) {
  const uint32_t st = c % kNeStages;
  const uint32_t r0 = c * RS, nr = nrows - r0 < RS ? nrows - r0 : RS;
  if (lane == 0) {
    mbar_expect_tx(&s_bar[st], nr * SW * 4u);
    s_live[st] = 1u;
  }
  __syncwarp();
  if (lane < nr)
    bulk_copy_g2s(s_stage + st * kNeStageWords + lane * SW, bits + (j0 + r0 + lane) * Wp + ws, SW * 4u, &s_bar[st]);
}

__global__ void __launch_bounds__(kNeThreads, 4) k_gmcr_ne(const uint32_t* __restrict__ bits, uint64_t Wp, uint64_t Qn,
                                                        const uint32_t* __restrict__ dgoff, uint32_t G, uint32_t GW, int prof,
                                                        uint32_t* __restrict__ NE) {
  extern __shared__ __align__(128) uint32_t s_stage[];  // kNeStages x kNeStageWords, then kNePadWords
  __shared__ __align__(8) uint64_t s_bar[kNeStages];
  __shared__ uint32_t s_live[kNeStages];  // stage holds (or receives) the chunk its next reader expects
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t g_lo = blockIdx.x * kNeThreads;
  const uint32_t g = g_lo + threadIdx.x;
  const uint32_t gw = g_lo / 32u + warp;
  NeLane L{};
  if (g < G) {
    const uint32_t s = dgoff[g], e = dgoff[g + 1];
    if (e > s) {
      L.i0 = s >> 5;
      L.nw = ((e + 31u) >> 5) - L.i0;
      L.mf = range_mask(L.i0, s, e, prof);
      L.ml = range_mask(L.i0 + L.nw - 1u, s, e, prof);
    }
  }
  L.m0 = L.nw ? L.mf : 0u;
  L.m1 = L.nw == 2u ? L.ml : (L.nw == 3u ? 0xFFFFFFFFu : 0u);
  L.m2 = L.nw == 3u ? L.ml : 0u;
  L.o1 = L.nw > 1u ? 1u : 0u;
  L.o2 = L.nw > 2u ? 2u : L.o1;
  const bool wide = !__all_sync(0xFFFFFFFFu, L.nw <= 3u);
  // the CTA's word span, 16-byte aligned at both ends (Wp is a multiple of 32)
  const uint32_t g_hi = g_lo + kNeThreads < G ? g_lo + kNeThreads : G;
  const uint32_t ws = (dgoff[g_lo] >> 5) & ~3u;
  uint32_t we = (((dgoff[g_hi] + 31u) >> 5) + 3u) & ~3u;
  if (we > Wp) we = static_cast<uint32_t>(Wp);
  const uint32_t SW = we > ws ? we - ws : 0u;
  const uint32_t rs_fit = SW ? kNeStageWords / SW : 0u;
  const uint32_t RS = rs_fit < 32u ? rs_fit : 32u;  // rows per stage (one copy per lane of warp 0)
  const bool staged = RS > 0u;
  const uint32_t a = L.nw ? L.i0 - ws : 0u;  // the lane's first word within a staged row
  const uint64_t j0 = static_cast<uint64_t>(blockIdx.y) * kNeRowsPerCta;
  const uint64_t j1 = j0 + kNeRowsPerCta < Qn ? j0 + kNeRowsPerCta : Qn;
  const uint32_t nrows = static_cast<uint32_t>(j1 - j0);
  const uint32_t nch = staged ? (nrows + RS - 1u) / RS : 1u;
  const uint32_t chunk_rows = staged ? RS : nrows;

  // warp 0 (lane 0's copy is the one used): stages whose phase lane 0 did not
  // see complete, and the parity of that phase
  uint32_t failed = 0, failed_par = 0;
  if (staged) {
    if (threadIdx.x == 0)
      for (uint32_t st = 0; st < kNeStages; ++st) {
        mbar_init(&s_bar[st], 1);
        s_live[st] = 0u;
      }
    __syncthreads();
    if (warp == 0)
      for (uint32_t c = 0; c < nch && c < kNeStages; ++c) ne_issue(c, lane, RS, SW, nrows, j0, ws, Wp, bits, s_stage, s_bar, s_live);
    __syncthreads();
  }
  uint32_t* ne_out = NE + j0 * GW + gw;
  for (uint32_t c = 0; c < nch; ++c) {
    const uint32_t st = c % kNeStages;
    const uint32_t r0 = c * chunk_rows;
    const uint32_t nr = nrows - r0 < chunk_rows ? nrows - r0 : chunk_rows;
    const bool live = staged && s_live[st];
    const bool have = live && mbar_wait_sleep(&s_bar[st], (c / kNeStages) & 1u, kNeSleepNs, kNePolls);
    const uint32_t* srow = s_stage + st * kNeStageWords + a;
    const uint32_t* grow = bits + (j0 + r0) * Wp + L.i0;
    // lane r keeps the NE word of the chunk's row r; the chunk's words are
    // stored together (one row per lane)
    uint32_t mine = 0;
    if (__all_sync(0xFFFFFFFFu, have) && !wide) {
      // words 1 and 2 are read even where the graph has fewer (masked to
      // zero; the ring has kNePadWords of slack past its end)
      const uint32_t* p = srow;
#pragma unroll 4
      for (uint32_t r = 0; r < nr; ++r, p += SW) {
        const uint32_t acc = (p[0] & L.m0) | (p[1] & L.m1) | (p[2] & L.m2);
        const uint32_t word = __ballot_sync(0xFFFFFFFFu, acc != 0u);
        mine = lane == r ? word : mine;
      }
    } else {
      for (uint32_t r = 0; r < nr; ++r) {
        const uint32_t* row = have ? srow + r * SW : grow + static_cast<uint64_t>(r) * Wp;
        const bool any = L.nw && (wide ? ne_any_wide(row, L) : ne_any_few(row, L));
        const uint32_t word = __ballot_sync(0xFFFFFFFFu, any);
        if (r < 32u) mine = lane == r ? word : mine;
        else if (lane == 0 && gw < GW) ne_out[static_cast<uint64_t>(r0 + r) * GW] = word;  // unstaged chunks only
      }
    }
    if (lane < nr && gw < GW) ne_out[static_cast<uint64_t>(r0 + lane) * GW] = mine;
    if (staged) {
      // once every warp is done with this stage, warp 0 refills it with chunk
      // c + kNeStages, unless lane 0 did not see a copy complete (then no
      // stage is refilled again and readers of the unfilled chunks, finding
      // s_live clear, read global memory)
      __syncthreads();
      if (warp == 0) {
        if (lane == 0 && live && !have) {
          failed |= 1u << st;
          failed_par |= ((c / kNeStages) & 1u) << st;
        }
        const bool stop = __shfl_sync(0xFFFFFFFFu, failed, 0) != 0u;
        if (c + kNeStages < nch && !stop) ne_issue(c + kNeStages, lane, RS, SW, nrows, j0, ws, Wp, bits, s_stage, s_bar, s_live);
        else if (lane == 0) s_live[st] = 0u;
      }
    }
  }
  // a copy whose wait ran out may still be in flight: wait for it again
  // (bounded) before the CTA's shared memory is released
  if (threadIdx.x == 0 && failed)
    for (uint32_t st = 0; st < kNeStages; ++st)
      if (failed >> st & 1u) mbar_wait_sleep(&s_bar[st], failed_par >> st & 1u, kNeSleepNs, kNePolls);
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

// Segment fill.  A warp owns 32 consecutive data graphs (one admission word
// column) and walks the query graphs 32 at a time: lane l loads the word of
// query q0 + l, then for each of the 32 graphs a vote gives the chunk's
// admitted queries in ascending order, which the lanes write to consecutive
// entries of that graph's segment (coalesced); lane j keeps graph j's write
// position.  Every segment is sorted.
__global__ void k_gmcr_fill(const uint32_t* __restrict__ admit, uint32_t GW, uint32_t QG, uint32_t G,
                            const uint32_t* __restrict__ offsets, uint32_t* __restrict__ indices,
                            uint32_t* __restrict__ pair_graph, uint64_t capacity) {
  const unsigned lane = threadIdx.x & 31u;
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t warp = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t gw = warp; gw < GW; gw += nwarps) {
    const uint32_t g_own = gw * 32u + lane;
    uint64_t cur = g_own < G ? offsets[g_own] : 0;  // lane j: next entry of graph gw * 32 + j
    const uint32_t in_tile = G - gw * 32u < 32u ? G - gw * 32u : 32u;
    for (uint32_t q0 = 0; q0 < QG; q0 += 32) {
      const uint32_t q = q0 + lane;
      const uint32_t w = q < QG ? admit[static_cast<uint64_t>(q) * GW + gw] : 0u;
      for (uint32_t j = 0; j < in_tile; ++j) {
        const uint32_t m = __ballot_sync(0xFFFFFFFFu, (w >> j) & 1u);
        if (!m) continue;
        const uint64_t base = __shfl_sync(0xFFFFFFFFu, cur, j);
        if ((m >> lane) & 1u) {
          const uint64_t pos = base + __popc(m & lt);
          if (pos < capacity) {
            indices[pos] = q;
            if (pair_graph) pair_graph[pos] = gw * 32u + j;
          }
        }
        if (lane == j) cur += __popc(m);
      }
    }
  }
}

}  // namespace

// The non-empty pass over the bitset into NE [Qn][GW].
static int launch_gmcr_ne(Queue* q, const Candidates* c, const Graph* data, uint64_t Qn, uint32_t* NE) {
  const uint32_t G = data->num_graphs;
  const uint32_t GW = (G + 31u) / 32u;
  const dim3 grid((G + kNeThreads - 1u) / kNeThreads, static_cast<unsigned>((Qn + kNeRowsPerCta - 1) / kNeRowsPerCta));
  if (grid.y > 65535u) return fail(SIGMO_ERR_DOMAIN, "too many query vertices (%llu)", static_cast<unsigned long long>(Qn));
  SIGMO_TRY(allow_max_dynamic_smem(reinterpret_cast<const void*>(k_gmcr_ne), q->device));
  k_gmcr_ne<<<grid, kNeThreads, kNeSmemBytes, q->stream>>>(c->bits, c->Wp, Qn, data->graph_offsets, G, GW, q->opts.profile, NE);
  return check_launch(q, "k_gmcr_ne");
}

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
    rc = launch_gmcr_ne(q, c, data, Qn, NE);
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
    SIGMO_TRY(launch_gmcr_ne(q, c, data, Qn, NE));
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
