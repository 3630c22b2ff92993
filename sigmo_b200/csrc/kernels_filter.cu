// Candidate-bitset kernels: the label filter (isomorphism.hpp:22-62), one
// refinement pass (isomorphism.hpp:64-127), the fused filter + R refinements
// of the batched form, and bitset reductions.
//
// Layout: row q (global query vertex) holds Wp uint32 words (the reference's
// W = ceil(N/32) rounded up to 32 words so every row starts 128-byte
// aligned); bit d%32 of word d/32 is candidate d (candidates.hpp:32-36).
// One thread owns one word (32 data vertices) and walks a chunk of rows, so
// the data-side operands of that word stay in registers / L1 while the row
// loop streams the bitset.
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

// filterCandidates: C[q][w] (|)= label match.
__global__ void k_filter(const uint8_t* __restrict__ qlab, uint64_t Qn, const uint8_t* __restrict__ dlab, uint64_t N,
                         uint64_t Wp, uint32_t* __restrict__ bits, int or_mode) {
  const uint64_t w = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (w >= Wp) return;
  LabelPlanes lp;
  load_label_planes(dlab, N, w, &lp);
  const uint64_t q0 = static_cast<uint64_t>(blockIdx.y) * kRowsPerBlock;
  const uint64_t q1 = q0 + kRowsPerBlock < Qn ? q0 + kRowsPerBlock : Qn;
  for (uint64_t q = q0; q < q1; ++q) {
    const uint32_t m = label_match(lp, qlab[q]);
    uint32_t* dst = bits + q * Wp + w;
    if (or_mode) *dst |= m;
    else *dst = m;
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

// Thermometer planes of the current data signatures: plane p = l*15 + (c-1)
// (l < 16, c = 1..15) has bit i of word w set when counter l of vertex 32w+i
// is >= c.  Warp per word, lane i = vertex 32w+i; planes are produced 32 at a
// time, lane j keeping plane (group + j) for one store.
__global__ void k_sig_thermo(const uint64_t* __restrict__ sig, uint64_t n, uint64_t Wp, uint32_t* __restrict__ therm) {
  const unsigned lane = threadIdx.x & 31u;
  const uint64_t warp = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
  const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
  for (uint64_t w = warp; w < Wp; w += nwarps) {
    const uint64_t v = w * 32 + lane;
    const uint64_t s = v < n ? sig[v] : 0ull;
    for (unsigned g0 = 0; g0 < 240; g0 += 32) {
      uint32_t mine = 0;
#pragma unroll
      for (unsigned j = 0; j < 32; ++j) {
        const unsigned p = g0 + j;
        if (p < 240) {
          const unsigned l = p / 15, c = p % 15 + 1;
          const uint32_t b = __ballot_sync(0xFFFFFFFFu, ((s >> (4 * l)) & 0xFu) >= c);
          if (lane == j) mine = b;
        }
      }
      if (g0 + lane < 240) therm[static_cast<uint64_t>(g0 + lane) * Wp + w] = mine;
    }
  }
}

// refineCandidates: C[q][w] &= AND over q's non-zero counters (l, c) of the
// thermometer plane "counter l >= c" of word w.  Rows are processed four at a
// time so four independent loads are in flight.
__global__ void k_refine(const uint64_t* __restrict__ qsig, uint64_t Qn, const uint32_t* __restrict__ therm, uint64_t Wp,
                         uint64_t W, uint32_t* __restrict__ bits) {
  const uint64_t w = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (w >= W) return;
  const uint64_t q0 = static_cast<uint64_t>(blockIdx.y) * kRowsPerBlock;
  const uint64_t q1 = q0 + kRowsPerBlock < Qn ? q0 + kRowsPerBlock : Qn;
  for (uint64_t q = q0; q < q1; q += 4) {
    uint32_t wd[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) wd[k] = (q + k < q1) ? bits[(q + k) * Wp + w] : 0u;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (!wd[k]) continue;
      const uint64_t qs = qsig[q + k];
      uint64_t nz = sig_nonzero_nibbles(qs);
      uint32_t m = wd[k];
      while (nz) {
        const uint32_t p = __ffsll(static_cast<long long>(nz)) - 1;  // 4 * label
        nz &= nz - 1;
        const uint32_t c = static_cast<uint32_t>((qs >> p) & 0xFu);
        m &= __ldg(therm + static_cast<uint64_t>((p >> 2) * 15 + c - 1) * Wp + w);
      }
      if (m != wd[k]) bits[(q + k) * Wp + w] = m;
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
  dim3 grid(grid_for(c->Wp, kWordsPerBlock), static_cast<unsigned>((c->rows + kRowsPerBlock - 1) / kRowsPerBlock));
  if (grid.y > 65535u) return fail(SIGMO_ERR_DOMAIN, "too many query vertices (%llu)", (unsigned long long)c->rows);
  k_filter<<<grid, kWordsPerBlock, 0, q->stream>>>(query->node_labels, c->rows, data->node_labels, data->total_nodes, c->Wp,
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

int launch_sig_thermo(Queue* q, const uint64_t* sig, uint64_t n, uint64_t Wp, uint32_t* therm) {
  if (!Wp) return SIGMO_OK;
  const unsigned threads = 256;
  k_sig_thermo<<<grid_for(Wp * 32, threads, 148u * 16u), threads, 0, q->stream>>>(sig, n, Wp, therm);
  return check_launch(q, "k_sig_thermo");
}

int launch_refine(Queue* q, const Graph* query, const Graph* data, const uint64_t* qsig, const uint32_t* therm,
                  Candidates* c) {
  (void)query;
  (void)data;
  if (!c->rows || !c->W) return SIGMO_OK;
  dim3 grid(grid_for(c->W, kWordsPerBlock), static_cast<unsigned>((c->rows + kRowsPerBlock - 1) / kRowsPerBlock));
  if (grid.y > 65535u) return fail(SIGMO_ERR_DOMAIN, "too many query vertices (%llu)", (unsigned long long)c->rows);
  k_refine<<<grid, kWordsPerBlock, 0, q->stream>>>(qsig, c->rows, therm, c->Wp, c->W, c->bits);
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
