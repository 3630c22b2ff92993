// Candidate-bitset kernels: the label filter (isomorphism.hpp:22-62), one
// refinement pass (isomorphism.hpp:64-127), the fused filter + R refinements
// of the batched form, and bitset reductions.
//
// Layout: row q (global query vertex) holds Wp uint32 words (the reference's
// W = ceil(N/32) rounded up to 32 words so every row starts 128-byte
// aligned); bit d%32 of word d/32 is candidate d (candidates.hpp:32-36).
// A thread owns a few consecutive words and walks a block of rows, so the
// data-side operands of those words stay in registers / shared memory while
// the row loop streams the bitset.
//
// Data signatures are bit-sliced per word: planes[l][w] is a uint4 whose
// component b has bit i set when bit b of counter l of vertex 32w+i is set.
// "every counter of q <= counter of d" for the 32 vertices of a word is then
// an AND over the query's non-zero counters of a 4-plane comparison against a
// constant, instead of 32 scalar comparisons.
#include <cuda_runtime.h>

#include "internal.hpp"

namespace sigmo_b200 {
namespace {

constexpr unsigned kWordsPerBlock = 128;
constexpr unsigned kRowsPerBlock = 64;

// Bit-sliced labels of the 32 vertices of word w.
struct LabelPlanes {
  uint32_t p[8];
  uint32_t valid;
};

__device__ __forceinline__ void load_label_planes(const uint8_t* __restrict__ lab, uint64_t N, uint64_t w, LabelPlanes* lp) {
#pragma unroll
  for (int b = 0; b < 8; ++b) lp->p[b] = 0;
  lp->valid = 0;
  const uint64_t base = w * 32ull;
  if (base >= N) return;
  uint8_t v[32];
  if (base + 32 <= N && ((reinterpret_cast<uintptr_t>(lab + base) & 15u) == 0)) {
    const uint4 a = *reinterpret_cast<const uint4*>(lab + base);
    const uint4 b = *reinterpret_cast<const uint4*>(lab + base + 16);
    *reinterpret_cast<uint4*>(v) = a;
    *reinterpret_cast<uint4*>(v + 16) = b;
    lp->valid = 0xFFFFFFFFu;
  } else {
    const uint32_t cnt = static_cast<uint32_t>(N - base < 32 ? N - base : 32);
#pragma unroll
    for (uint32_t i = 0; i < 32; ++i) v[i] = i < cnt ? lab[base + i] : 0;
    lp->valid = cnt >= 32 ? 0xFFFFFFFFu : ((1u << cnt) - 1u);
  }
#pragma unroll
  for (uint32_t i = 0; i < 32; ++i) {
#pragma unroll
    for (int b = 0; b < 8; ++b) lp->p[b] |= static_cast<uint32_t>((v[i] >> b) & 1u) << i;
  }
}

// Vertices of the word whose label equals ql, or all if ql is the wildcard.
__device__ __forceinline__ uint32_t label_match(const LabelPlanes& lp, uint8_t ql) {
  if (ql == kWildcard) return lp.valid;
  uint32_t m = lp.valid;
#pragma unroll
  for (int b = 0; b < 8; ++b) m &= ((ql >> b) & 1u) ? lp.p[b] : ~lp.p[b];
  return m;
}

// AND of "counter l of d >= counter l of q" over the non-zero counters of q.
__device__ __forceinline__ uint32_t dominance_word(uint64_t qs, const uint4* __restrict__ planes, uint64_t Wp, uint64_t w,
                                                   uint32_t m) {
  uint64_t nz = sig_nonzero_nibbles(qs);
  while (nz && m) {
    const uint32_t p = __ffsll(static_cast<long long>(nz)) - 1;  // 4 * label
    nz &= nz - 1;
    const uint32_t c = static_cast<uint32_t>((qs >> p) & 0xFu);
    const uint4 P = __ldg(planes + static_cast<uint64_t>(p >> 2) * Wp + w);
    m &= ge_sliced(P.x, P.y, P.z, P.w, c);
  }
  return m;
}

// The row-block kernels below (k_filter, k_refine) give a block kTabRows
// consecutive rows (query vertices) and a span of words; the rows of a block
// use few distinct labels / (label, count) thresholds, so each thread first
// evaluates those once for its words into a shared-memory table, and the row
// loop is then a table read, the bitset access and nothing else.
constexpr unsigned kTabThreads = 128;
constexpr unsigned kTabRows = 64;
constexpr unsigned kFilterSlots = 16;   // distinct labels tabulated per block
constexpr unsigned kRefineSlots = 32;   // distinct (label, count) thresholds tabulated per block
constexpr uint16_t kNoSlot = 0x8000u;   // row entry computed directly (beyond the table)

// Exclusive ranks of the set bits of a shared bitmap of `nwords` words (<= 32),
// computed by warp 0: rank_of[bit] = rank, or 0xFF beyond `cap`; item_of[rank]
// = bit for ranks below cap; *count = min(total, cap).
__device__ __forceinline__ void rank_bits(const uint32_t* present, unsigned nwords, uint8_t* rank_of, uint8_t* item_of,
                                          unsigned cap, uint32_t* count) {
  const unsigned lane = threadIdx.x;
  uint32_t word = lane < nwords ? present[lane] : 0u;
  const uint32_t cnt = __popc(word);
  uint32_t incl = cnt;
#pragma unroll
  for (unsigned o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= o) incl += t;
  }
  uint32_t rank = incl - cnt;
  while (word) {
    const uint32_t b = __ffs(word) - 1;
    word &= word - 1;
    const uint32_t item = lane * 32u + b;
    rank_of[item] = rank < cap ? static_cast<uint8_t>(rank) : 0xFFu;
    if (rank < cap) item_of[rank] = static_cast<uint8_t>(item);
    ++rank;
  }
  if (lane == 31) *count = incl < cap ? incl : cap;
}

// filterCandidates: C[q][w] (|)= label match.  Thread t owns the four words
// 4t..4t+3 of the block's 512-word span (one 16-byte access per row).
__global__ void __launch_bounds__(kTabThreads) k_filter(const uint8_t* __restrict__ qlab, uint64_t Qn,
                                                        const uint8_t* __restrict__ dlab, uint64_t N, uint64_t Wp,
                                                        uint32_t* __restrict__ bits, int or_mode) {
  __shared__ uint32_t present[8];
  __shared__ uint8_t slot_of[256];
  __shared__ uint8_t slot_label[kFilterSlots];
  __shared__ uint32_t nslots;
  __shared__ uint8_t row_slot[kTabRows];
  __shared__ uint4 T[kFilterSlots][kTabThreads];
  const unsigned tid = threadIdx.x;
  const uint64_t w0 = (static_cast<uint64_t>(blockIdx.x) * kTabThreads + tid) * 4u;
  const uint64_t q0 = static_cast<uint64_t>(blockIdx.y) * kTabRows;
  const uint32_t nrows = static_cast<uint32_t>(Qn - q0 < kTabRows ? Qn - q0 : kTabRows);
  if (tid < 8) present[tid] = 0;
  __syncthreads();
  uint8_t ql = 0;
  if (tid < nrows) {
    ql = qlab[q0 + tid];
    atomicOr(&present[ql >> 5], 1u << (ql & 31u));
  }
  __syncthreads();
  if (tid < 32) rank_bits(present, 8, slot_of, slot_label, kFilterSlots, &nslots);
  __syncthreads();
  if (tid < nrows) row_slot[tid] = slot_of[ql];
  const bool in = w0 < Wp;  // Wp is a multiple of 32, so all four words are in the row
  LabelPlanes lp[4];
  if (in) {
#pragma unroll
    for (int k = 0; k < 4; ++k) load_label_planes(dlab, N, w0 + k, &lp[k]);
  }
  for (uint32_t sl = 0; sl < nslots; ++sl) {
    const uint8_t l = slot_label[sl];
    uint4 v = make_uint4(0, 0, 0, 0);
    if (in) v = make_uint4(label_match(lp[0], l), label_match(lp[1], l), label_match(lp[2], l), label_match(lp[3], l));
    T[sl][tid] = v;
  }
  __syncthreads();
  if (!in) return;
  for (uint32_t r = 0; r < nrows; ++r) {
    const uint8_t sl = row_slot[r];
    uint4 m;
    if (sl != 0xFFu) {
      m = T[sl][tid];
    } else {
      const uint8_t l = qlab[q0 + r];
      m = make_uint4(label_match(lp[0], l), label_match(lp[1], l), label_match(lp[2], l), label_match(lp[3], l));
    }
    uint4* dst = reinterpret_cast<uint4*>(bits + (q0 + r) * Wp + w0);
    if (or_mode) {
      const uint4 o = *dst;
      m.x |= o.x;
      m.y |= o.y;
      m.z |= o.z;
      m.w |= o.w;
    }
    *dst = m;
  }
}

// Bit-slice signatures: warp per word, lane i = vertex 32w+i.
__global__ void k_sig_planes(const uint64_t* __restrict__ sig, uint64_t n, uint64_t Wp, uint4* __restrict__ planes) {
  const unsigned lane = threadIdx.x & 31u;
  const uint64_t warp = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
  const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
  for (uint64_t w = warp; w < Wp; w += nwarps) {
    const uint64_t v = w * 32 + lane;
    const uint64_t s = v < n ? sig[v] : 0ull;
    uint4 mine = make_uint4(0, 0, 0, 0);
#pragma unroll
    for (unsigned l = 0; l < 16; ++l) {
      const uint32_t x0 = __ballot_sync(0xFFFFFFFFu, (s >> (4 * l)) & 1ull);
      const uint32_t x1 = __ballot_sync(0xFFFFFFFFu, (s >> (4 * l + 1)) & 1ull);
      const uint32_t x2 = __ballot_sync(0xFFFFFFFFu, (s >> (4 * l + 2)) & 1ull);
      const uint32_t x3 = __ballot_sync(0xFFFFFFFFu, (s >> (4 * l + 3)) & 1ull);
      if (lane == l) mine = make_uint4(x0, x1, x2, x3);
    }
    if (lane < 16) planes[static_cast<uint64_t>(lane) * Wp + w] = mine;
  }
}

// refineCandidates: C[q][w] &= AND over q's non-zero counters (l, c) of
// "counter l of vertex >= c", evaluated from the bit-sliced data signatures
// (planes[l][w], see k_sig_planes).  Thread t owns the two words 2t, 2t+1 of
// the block's 256-word span; the block's distinct thresholds (kRefineSlots at
// most, about ten for molecule queries) are tabulated per thread, and a word
// is written back only when it changed.
__device__ __forceinline__ uint2 ge_pair(const uint4* __restrict__ planes, uint64_t Wp, uint64_t w0, uint32_t p) {
  const uint32_t l = p / 15u, c = p % 15u + 1u;
  const uint4 a = __ldg(planes + static_cast<uint64_t>(l) * Wp + w0);
  const uint4 b = __ldg(planes + static_cast<uint64_t>(l) * Wp + w0 + 1);
  return make_uint2(ge_sliced(a.x, a.y, a.z, a.w, c), ge_sliced(b.x, b.y, b.z, b.w, c));
}

__global__ void __launch_bounds__(kTabThreads) k_refine(const uint64_t* __restrict__ qsig, uint64_t Qn,
                                                        const uint4* __restrict__ planes, uint64_t Wp,
                                                        uint32_t* __restrict__ bits) {
  __shared__ uint32_t present[8];  // threshold p = 15 l + c - 1 (240 bits)
  __shared__ uint8_t slot_of[256];
  __shared__ uint8_t slot_p[kRefineSlots];
  __shared__ uint32_t nslots;
  __shared__ uint8_t row_cnt[kTabRows];
  __shared__ uint16_t row_ent[kTabRows][16];
  __shared__ uint2 T[kRefineSlots][kTabThreads];
  const unsigned tid = threadIdx.x;
  const uint64_t w0 = (static_cast<uint64_t>(blockIdx.x) * kTabThreads + tid) * 2u;
  const uint64_t q0 = static_cast<uint64_t>(blockIdx.y) * kTabRows;
  const uint32_t nrows = static_cast<uint32_t>(Qn - q0 < kTabRows ? Qn - q0 : kTabRows);
  if (tid < 8) present[tid] = 0;
  __syncthreads();
  uint64_t qs = 0;
  if (tid < nrows) {
    qs = qsig[q0 + tid];
    for (uint32_t l = 0; l < 16; ++l) {
      const uint32_t c = static_cast<uint32_t>((qs >> (4 * l)) & 0xFu);
      if (c) {
        const uint32_t p = 15u * l + c - 1u;
        atomicOr(&present[p >> 5], 1u << (p & 31u));
      }
    }
  }
  __syncthreads();
  if (tid < 32) rank_bits(present, 8, slot_of, slot_p, kRefineSlots, &nslots);
  __syncthreads();
  if (tid < nrows) {
    uint32_t k = 0;
    for (uint32_t l = 0; l < 16; ++l) {
      const uint32_t c = static_cast<uint32_t>((qs >> (4 * l)) & 0xFu);
      if (c) {
        const uint32_t p = 15u * l + c - 1u;
        const uint8_t sl = slot_of[p];
        row_ent[tid][k++] = sl != 0xFFu ? sl : static_cast<uint16_t>(kNoSlot | p);
      }
    }
    row_cnt[tid] = static_cast<uint8_t>(k);
  }
  const bool in = w0 < Wp;  // Wp is a multiple of 32, so both words are in the row
  for (uint32_t sl = 0; sl < nslots; ++sl) T[sl][tid] = in ? ge_pair(planes, Wp, w0, slot_p[sl]) : make_uint2(0, 0);
  __syncthreads();
  if (!in) return;
  constexpr uint32_t kBatch = 8;  // rows whose words are loaded before any is processed
  for (uint32_t r0 = 0; r0 < nrows; r0 += kBatch) {
    uint2 wd[kBatch];
#pragma unroll
    for (uint32_t k = 0; k < kBatch; ++k)
      wd[k] = r0 + k < nrows ? *reinterpret_cast<const uint2*>(bits + (q0 + r0 + k) * Wp + w0) : make_uint2(0, 0);
#pragma unroll
    for (uint32_t k = 0; k < kBatch; ++k) {
      const uint32_t r = r0 + k;
      if (r >= nrows || !(wd[k].x | wd[k].y)) continue;
      uint2 m = wd[k];
      const uint32_t n = row_cnt[r];
      for (uint32_t e = 0; e < n; ++e) {
        const uint16_t ent = row_ent[r][e];
        const uint2 t = ent < kNoSlot ? T[ent][tid] : ge_pair(planes, Wp, w0, ent & 0xFFu);
        m.x &= t.x;
        m.y &= t.y;
      }
      if (m.x != wd[k].x || m.y != wd[k].y) *reinterpret_cast<uint2*>(bits + (q0 + r) * Wp + w0) = m;
    }
  }
}

// Batched form: C[q][w] = label match AND dominance at every iteration
// r = 1..R (qsig_all [R][Qn], planes_all [R][16][Wp]); the final bitset of
// the reference's filter + R refinements, written once.
__global__ void k_fused_filter(const uint8_t* __restrict__ qlab, const uint64_t* __restrict__ qsig_all, uint64_t Qn,
                               const uint8_t* __restrict__ dlab, uint64_t N, const uint4* __restrict__ planes_all,
                               uint64_t Wp, uint32_t R, uint32_t* __restrict__ bits) {
  const uint64_t w = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (w >= Wp) return;
  LabelPlanes lp;
  load_label_planes(dlab, N, w, &lp);
  const uint64_t q0 = static_cast<uint64_t>(blockIdx.y) * kRowsPerBlock;
  const uint64_t q1 = q0 + kRowsPerBlock < Qn ? q0 + kRowsPerBlock : Qn;
  for (uint64_t q = q0; q < q1; ++q) {
    uint32_t m = label_match(lp, qlab[q]);
    for (uint32_t r = 0; r < R && m; ++r)
      m = dominance_word(qsig_all[static_cast<uint64_t>(r) * Qn + q], planes_all + static_cast<uint64_t>(r) * 16 * Wp, Wp, w, m);
    bits[q * Wp + w] = m;
  }
}

// getCandidatesCount(source) per row (candidates.hpp:77-81).
__global__ void k_row_counts(const uint32_t* __restrict__ bits, uint64_t rows, uint64_t W, uint64_t Wp,
                             uint32_t* __restrict__ counts) {
  for (uint64_t r = blockIdx.x; r < rows; r += gridDim.x) {
    uint32_t c = 0;
    for (uint64_t w = threadIdx.x; w < W; w += blockDim.x) c += __popc(bits[r * Wp + w]);
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
    __shared__ uint32_t part[32];
    if ((threadIdx.x & 31u) == 0) part[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x < 32) {
      c = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0u;
      for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
      if (threadIdx.x == 0) counts[r] = c;
    }
    __syncthreads();
  }
}

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// digest = sum_q mix64(h_q + q * K2), h_q = sum_w mix64(word ^ (w * K1)), over
// the reference layout's W words (mod 2^64).
__global__ void k_digest(const uint32_t* __restrict__ bits, uint64_t rows, uint64_t W, uint64_t Wp,
                         unsigned long long* __restrict__ out) {
  const uint64_t K1 = 0x9E3779B97F4A7C15ull, K2 = 0xC2B2AE3D27D4EB4Full;
  for (uint64_t r = blockIdx.x; r < rows; r += gridDim.x) {
    uint64_t h = 0;
    for (uint64_t w = threadIdx.x; w < W; w += blockDim.x) h += mix64(static_cast<uint64_t>(bits[r * Wp + w]) ^ (w * K1));
    for (int o = 16; o; o >>= 1) h += __shfl_xor_sync(0xFFFFFFFFu, h, o);
    __shared__ uint64_t part[32];
    if ((threadIdx.x & 31u) == 0) part[threadIdx.x >> 5] = h;
    __syncthreads();
    if (threadIdx.x < 32) {
      h = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0ull;
      for (int o = 16; o; o >>= 1) h += __shfl_xor_sync(0xFFFFFFFFu, h, o);
      if (threadIdx.x == 0) atomicAdd(out, static_cast<unsigned long long>(mix64(h + r * K2)));
    }
    __syncthreads();
  }
}

}  // namespace

int launch_filter(Queue* q, const Graph* query, const Graph* data, Candidates* c) {
  if (!c->rows || !c->Wp) return SIGMO_OK;
  dim3 grid(grid_for(c->Wp, 4u * kTabThreads), static_cast<unsigned>((c->rows + kTabRows - 1) / kTabRows));
  if (grid.y > 65535u) return fail(SIGMO_ERR_DOMAIN, "too many query vertices (%llu)", (unsigned long long)c->rows);
  k_filter<<<grid, kTabThreads, 0, q->stream>>>(query->node_labels, c->rows, data->node_labels, data->total_nodes, c->Wp,
                                                c->bits, c->known_zero ? 0 : 1);
  c->known_zero = false;
  return check_launch(q, "k_filter");
}

int launch_sig_planes(Queue* q, const uint64_t* sig, uint64_t n, uint64_t Wp, uint32_t* planes) {
  if (!Wp) return SIGMO_OK;
  const unsigned threads = 256;
  k_sig_planes<<<grid_for(Wp * 32, threads, 148u * 16u), threads, 0, q->stream>>>(sig, n, Wp, reinterpret_cast<uint4*>(planes));
  return check_launch(q, "k_sig_planes");
}

int launch_refine(Queue* q, const uint64_t* qsig, const uint32_t* planes, Candidates* c) {
  if (!c->rows || !c->W) return SIGMO_OK;
  dim3 grid(grid_for(c->Wp, 2u * kTabThreads), static_cast<unsigned>((c->rows + kTabRows - 1) / kTabRows));
  if (grid.y > 65535u) return fail(SIGMO_ERR_DOMAIN, "too many query vertices (%llu)", (unsigned long long)c->rows);
  k_refine<<<grid, kTabThreads, 0, q->stream>>>(qsig, c->rows, reinterpret_cast<const uint4*>(planes), c->Wp, c->bits);
  return check_launch(q, "k_refine");
}

int launch_fused_filter(Queue* q, const Graph* query, const Graph* data, uint32_t R, const uint64_t* qsig_all,
                        const uint32_t* planes_all, Candidates* c) {
  if (!c->rows || !c->Wp) return SIGMO_OK;
  dim3 grid(grid_for(c->Wp, kWordsPerBlock), static_cast<unsigned>((c->rows + kRowsPerBlock - 1) / kRowsPerBlock));
  if (grid.y > 65535u) return fail(SIGMO_ERR_DOMAIN, "too many query vertices (%llu)", (unsigned long long)c->rows);
  k_fused_filter<<<grid, kWordsPerBlock, 0, q->stream>>>(query->node_labels, qsig_all, c->rows, data->node_labels,
                                                         data->total_nodes, reinterpret_cast<const uint4*>(planes_all), c->Wp,
                                                         R, c->bits);
  c->known_zero = false;
  return check_launch(q, "k_fused_filter");
}

// Fused filter over the first `Wstride` words of every row into a bitset of
// that row stride (the batched form materialises only the words its literal
// join reads).
int launch_fused_filter_raw(Queue* q, const uint8_t* qlab, const uint64_t* qsig_all, uint64_t Qn, const uint8_t* dlab,
                            uint64_t N, const uint32_t* planes_all, uint64_t Wstride, uint32_t R, uint32_t* bits) {
  if (!Qn || !Wstride) return SIGMO_OK;
  dim3 grid(grid_for(Wstride, kWordsPerBlock), static_cast<unsigned>((Qn + kRowsPerBlock - 1) / kRowsPerBlock));
  if (grid.y > 65535u) return fail(SIGMO_ERR_DOMAIN, "too many query vertices (%llu)", (unsigned long long)Qn);
  k_fused_filter<<<grid, kWordsPerBlock, 0, q->stream>>>(qlab, qsig_all, Qn, dlab, N, reinterpret_cast<const uint4*>(planes_all),
                                                         Wstride, R, bits);
  return check_launch(q, "k_fused_filter");
}

int launch_row_counts(Queue* q, const Candidates* c, uint32_t* d_counts) {
  if (!c->rows) return SIGMO_OK;
  k_row_counts<<<grid_for(c->rows, 1, 148u * 64u), 256, 0, q->stream>>>(c->bits, c->rows, c->W, c->Wp, d_counts);
  return check_launch(q, "k_row_counts");
}

int launch_digest(Queue* q, const Candidates* c, uint64_t* d_digest) {
  SIGMO_CUDA_TRY(cudaMemsetAsync(d_digest, 0, sizeof(uint64_t), q->stream));
  if (!c->rows) return SIGMO_OK;
  k_digest<<<grid_for(c->rows, 1, 148u * 64u), 256, 0, q->stream>>>(c->bits, c->rows, c->W, c->Wp,
                                                                    reinterpret_cast<unsigned long long*>(d_digest));
  return check_launch(q, "k_digest");
}

}  // namespace sigmo_b200
