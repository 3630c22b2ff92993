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

// Step budget (JoinLimit): a lane counts the DFS levels it leaves; past the
// budget it raises the status word and stops.  Lanes check the word before
// taking more work, so a spent budget ends the launch soon after.
__device__ __forceinline__ bool budget_spent(const JoinLimit& lim, uint64_t& steps) {
  if (lim.budget && ++steps > lim.budget) {
    atomicOr(lim.status, kJoinStatusBudget);
    return true;
  }
  return false;
}
__device__ __forceinline__ bool join_stopped(const JoinLimit& lim) {
  return lim.budget && *reinterpret_cast<volatile const unsigned int*>(lim.status) != 0u;
}

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

// Per-pair cache of the range-masked candidate words of every query vertex
// (a data graph of <= 64 vertices spans at most 3 bitset words), so the DFS's
// repeated getCandidatesCount / getCandidateAt read registers/L1 instead of
// the bitset.  Values are exactly those of candidates.hpp:86-162.
struct PairCands {
  uint32_t w[kMaxQueryNodes][3];
  uint32_t cnt[kMaxQueryNodes];
  uint32_t i0, nw;
  __device__ __forceinline__ void load(const uint32_t* __restrict__ bits, uint64_t Wp, uint32_t qoff, uint32_t n, uint32_t s,
                                       uint32_t e, int prof) {
    i0 = s >> 5;
    nw = ((e + 31u) >> 5) - i0;
    for (uint32_t j = 0; j < n; ++j) {
      const uint32_t* row = bits + static_cast<uint64_t>(qoff + j) * Wp;
      uint32_t c = 0;
      for (uint32_t k = 0; k < 3; ++k) {
        const uint32_t v = k < nw ? (row[i0 + k] & range_mask(i0 + k, s, e, prof)) : 0u;
        w[j][k] = v;
        c += __popc(v);
      }
      cnt[j] = c;
    }
  }
  __device__ __forceinline__ uint32_t at(uint32_t j, uint32_t idx) const {
    uint32_t c = 0;
    for (uint32_t k = 0; k < nw; ++k) {
      uint32_t blk = w[j][k];
      const uint32_t bc = __popc(blk);
      if (c + bc > idx) {
        while (blk) {
          const uint32_t t = __ffs(blk) - 1;
          if (c == idx) return ((i0 + k) << 5) + t;
          blk &= blk - 1;
          ++c;
        }
      } else {
        c += bc;
      }
    }
    return 0xFFFFFFFFu;
  }
};

template <bool EXACT>
__global__ void k_join_literal(const uint32_t* __restrict__ bits, uint64_t Wp, int prof,
                               const uint32_t* __restrict__ qgoff, const uint64_t* __restrict__ qadj,
                               const uint32_t* __restrict__ dgoff, const uint64_t* __restrict__ dadj, uint32_t dAW,
                               const uint32_t* __restrict__ droff, const uint32_t* __restrict__ dcol,
                               const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ indices, uint32_t g0,
                               uint32_t g1, uint32_t q_begin, uint32_t q_end, int find_first, uint64_t* __restrict__ counts,
                               unsigned long long* __restrict__ d_total, JoinLimit lim) {
  const uint32_t wg = blockDim.x, lid = threadIdx.x;
  uint64_t my_total = 0;
  uint64_t steps = 0;
  bool stop = false;
  PairCands pc;
  uint64_t rowc[kMaxQueryNodes];   // adjacency row of mapping[i] (graphs <= 64 vertices)
  uint64_t vmask[kMaxQueryNodes];  // candidates passing isValidMapping at depth d (graphs <= 64 vertices)
  for (uint32_t g = g0 + blockIdx.x; g < g1; g += gridDim.x) {
    const uint32_t s = dgoff[g], e = dgoff[g + 1], ng = e - s;
    const bool small = ng <= 64u;
    // the segment's slots whose query graph is in [q_begin, q_end) (segments
    // are sorted by query graph, so they are contiguous)
    uint32_t seg0 = offsets[g], seg1 = offsets[g + 1];
    if (q_begin != 0 || q_end != 0xFFFFFFFFu) {
      uint32_t lo = seg0, hi = seg1;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (indices[mid] < q_begin) lo = mid + 1;
        else hi = mid;
      }
      uint32_t lo2 = lo, hi2 = seg1;
      while (lo2 < hi2) {
        const uint32_t mid = (lo2 + hi2) >> 1;
        if (indices[mid] < q_end) lo2 = mid + 1;
        else hi2 = mid;
      }
      seg0 = lo;
      seg1 = lo2;
    }
    const uint32_t seglen = seg1 - seg0;
    uint32_t mapping[kMaxQueryNodes + 1];
#pragma unroll 1
    for (uint32_t k = 0; k <= kMaxQueryNodes; ++k) mapping[k] = 0;
    for (uint32_t it = lid; it < seglen; it += wg) {
      if (join_stopped(lim)) {
        stop = true;
        break;
      }
      const uint32_t qg = indices[seg0 + it];
      const uint32_t qoff = qgoff[qg], n = qgoff[qg + 1] - qoff;
      if (small) pc.load(bits, Wp, qoff, n, s, e, prof);
      auto count_of = [&](uint32_t qn) -> uint32_t {
        return small ? pc.cnt[qn] : cand_count(bits + static_cast<uint64_t>(qoff + qn) * Wp, s, e, prof);
      };
      auto cand_of = [&](uint32_t qn, uint32_t idx) -> uint32_t {
        return small ? pc.at(qn, idx) : cand_at(bits + static_cast<uint64_t>(qoff + qn) * Wp, idx, s, e, prof);
      };
      // isValidMapping (isomorphism.hpp:150-168).  Its result depends only on
      // mapping[0..qn-1], which stay fixed while the frame at depth qn runs, so
      // for graphs of <= 64 vertices it is evaluated once per push as the bit
      // set vmask[qn] and each candidate is then one bit test.
      auto valid = [&](uint32_t qn, uint32_t cand) -> bool {
        if (small) return (vmask[qn] >> (cand - s)) & 1ull;
        const uint64_t qrow_bit = 1ull << qn;
        for (uint32_t i = 0; i < qn; ++i) {
          const bool qa = (qadj[qoff + i] & qrow_bit) != 0;
          if (qa != data_neighbor(mapping[i], cand, s, ng, dadj, dAW, droff, dcol)) return false;
        }
        return true;
      };
      // vmask[d] from rowc[0..d-1]: local t is valid iff for every i < d,
      // (d in query row i) == (t in data row of mapping[i]).
      auto push_mask = [&](uint32_t d) {
        if (!small || d >= n) return;
        uint64_t vm = ~0ull;
        const uint64_t qbit = 1ull << d;
        for (uint32_t i = 0; i < d; ++i) vm &= ((qadj[qoff + i] & qbit) ? rowc[i] : ~rowc[i]);
        vmask[d] = vm;
      };
      if (small) vmask[0] = ~0ull;
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
          if (small && qn + 1 == n && fr.idx == 0) {
            // The last level in one step (graphs of <= 64 vertices).  Its
            // candidates are distinct local bits, so placing one never hides a
            // later one, and valid() does not read `visited`: the frame finds
            // popc(candidates & valid & ~visited), sets the bits of those below
            // vertex 256 (refbit gives none above), leaves mapping[n - 1] at the
            // last one placed (the first under find-first, which stops there),
            // then is used up -- what the candidate-by-candidate loop does.
            const uint32_t sh = s & 31u;
            const uint64_t lo = static_cast<uint64_t>(pc.w[qn][0]) | (static_cast<uint64_t>(pc.w[qn][1]) << 32);
            const uint64_t cm = (lo >> sh) | (sh ? (static_cast<uint64_t>(pc.w[qn][2]) << (64u - sh)) : 0ull);
            // REF_X86: every local bit is live (a <= 64-vertex graph's set is exact)
            const uint64_t low = prof == kProfileX86 ? ~0ull
                                 : (s >= 256u ? 0ull : (256u - s >= 64u ? ~0ull : ((1ull << (256u - s)) - 1ull)));
            uint64_t place = cm & vmask[qn] & ~visited;
            if (place) {
              if (find_first) place &= 0ull - place;
              found += __popcll(place);
              visited |= place & low;
              mapping[qn] = s + 63u - static_cast<uint32_t>(__clzll(static_cast<long long>(place)));
              if (find_first) break;
            }
            --top;
            visited &= ~refbit_prof(mapping[qn], s, prof);
            if (top == 1) visited = 0;
            if (budget_spent(lim, steps)) {
              stop = true;
              break;
            }
            continue;
          }
          if (fr.idx >= count_of(qn)) {
            --top;
            visited &= ~refbit_prof(mapping[qn], s, prof);
            if (top == 1) visited = 0;
            if (budget_spent(lim, steps)) {
              stop = true;
              break;
            }
            continue;
          }
          const uint32_t cand = cand_of(qn, fr.idx);
          stack[top - 1].idx++;
          if (visited & refbit_prof(cand, s, prof)) continue;
          if (valid(qn, cand)) {
            mapping[qn] = cand;
            if (small) rowc[qn] = dadj[static_cast<uint64_t>(cand) * dAW];
            visited |= refbit_prof(cand, s, prof);
            stack[top++] = {qn + 1, 0u};
            push_mask(qn + 1);
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
          if (fr.idx >= count_of(qn)) {
            --top;
            if (budget_spent(lim, steps)) {
              stop = true;
              break;
            }
            continue;
          }
          const uint32_t cand = cand_of(qn, fr.idx);
          stack[top - 1].idx++;
          const uint32_t t = cand - s;
          if ((used[t >> 6] >> (t & 63u)) & 1ull) continue;
          if (valid(qn, cand)) {
            mapping[qn] = cand;
            if (small) rowc[qn] = dadj[static_cast<uint64_t>(cand) * dAW];
            placed[qn] = cand;
            used[t >> 6] |= 1ull << (t & 63u);
            stack[top++] = {qn + 1, 0u};
            push_mask(qn + 1);
          }
        }
      }
      if (stop) break;
      counts[seg0 + it] = found;
      my_total += found;
    }
    if (stop) break;
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

// k_join_literal for its common case: every data graph of the launch has at
// most 64 vertices and every query at most kLitLevels.  The same DFS, step for
// step, with the per-level state of each thread in shared memory
// ([level][thread], no local-memory stack):
//   cm[j]   the pair's range-masked candidates of query vertex j as graph-local
//           bits (candidates.hpp:86-162; at most 3 bitset words per graph);
//   rem[j]  the candidates the frame at depth j has still to try, taken in
//           ascending order like getCandidateAt(idx) for idx = 0, 1, ...
//           Only those passing isValidMapping are kept (its result depends on
//           mapping[0..j-1], fixed while the frame runs, so it is one AND
//           when the frame is pushed); the others are skipped by the
//           reference with no effect, so the placements are the same;
//   map[j]  mapping[j] as a local id, carried across the thread's pairs of a
//           data graph like the reference's private array (isomorphism.hpp:309);
//           a fresh work-item's mapping[] holds global vertex 0, which is
//           local 0 of a graph starting at vertex 0 and kLitOutside (no
//           bit of the graph) otherwise.
// REF_PTX keeps the reference's `visited` bookkeeping (utils.hpp:64-96,
// isomorphism.hpp:346-369): a frame that runs out unsets only mapping[depth]
// (perhaps stale), and the set is cleared when the DFS is back at depth 0.
// EXACT runs the injective DFS: the pick of a frame is unset when its child
// frame runs out.  The last query vertex is placed in one step, as in
// k_join_literal.
constexpr uint32_t kLitLevels = 32;
constexpr uint8_t kLitOutside = 0xFFu;
// 17 B per level and thread: 68 KB for the default 128 threads, so a block
// fits beside two persistent k_join_masks CTAs on one SM.
constexpr size_t kLitBytesPerThread = kLitLevels * (2 * sizeof(uint64_t) + 1);

template <bool EXACT>
__global__ void k_join_literal_small(const uint32_t* __restrict__ bits, uint64_t Wp, int prof,
                                     const uint32_t* __restrict__ qgoff, const uint64_t* __restrict__ qadj,
                                     const uint32_t* __restrict__ dgoff, const uint64_t* __restrict__ dadj, uint32_t dAW,
                                     const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ indices, uint32_t g0,
                                     uint32_t g1, uint32_t q_begin, uint32_t q_end, int find_first,
                                     uint64_t* __restrict__ counts, unsigned long long* __restrict__ d_total, JoinLimit lim) {
  extern __shared__ uint64_t lit_sm[];
  const uint32_t wg = blockDim.x, lid = threadIdx.x;
  uint64_t* cm = lit_sm;
  uint64_t* rem = lit_sm + kLitLevels * wg;
  uint8_t* map = reinterpret_cast<uint8_t*>(lit_sm + 2 * kLitLevels * wg);
#define LV(arr, l) arr[(l) * wg + lid]
  uint64_t my_total = 0, steps = 0;
  bool stop = false;
  for (uint32_t g = g0 + blockIdx.x; g < g1 && !stop; g += gridDim.x) {
    const uint32_t s = dgoff[g], e = dgoff[g + 1];
    uint32_t seg0 = offsets[g], seg1 = offsets[g + 1];
    if (q_begin != 0 || q_end != 0xFFFFFFFFu) {  // the segment's slots with query graph in [q_begin, q_end)
      uint32_t lo = seg0, hi = seg1;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (indices[mid] < q_begin) lo = mid + 1;
        else hi = mid;
      }
      uint32_t lo2 = lo, hi2 = seg1;
      while (lo2 < hi2) {
        const uint32_t mid = (lo2 + hi2) >> 1;
        if (indices[mid] < q_end) lo2 = mid + 1;
        else hi2 = mid;
      }
      seg0 = lo;
      seg1 = lo2;
    }
    const uint8_t map0 = s == 0 ? 0 : kLitOutside;
#pragma unroll 1
    for (uint32_t k = 0; k < kLitLevels; ++k) LV(map, k) = map0;  // mapping[] of a fresh work-item
    // graph-local bits the reference's uint8-indexed visited set can hold:
    // under REF_PTX those whose global id is below 256; under REF_X86 all
    // (the count modulo 64 is the local id).  A fresh work-item's mapping[]
    // (global vertex 0) names under REF_X86 the bit (0 - s) mod 64.
    const uint64_t low = prof == kProfileX86 ? ~0ull
                         : (s >= 256u ? 0ull : (256u - s >= 64u ? ~0ull : ((1ull << (256u - s)) - 1ull)));
    const uint64_t outside_bit = prof == kProfileX86 ? (1ull << ((0u - s) & 63u)) : 0ull;
    const uint32_t i0 = s >> 5, nw = ((e + 31u) >> 5) - i0, sh = s & 31u;
    for (uint32_t it = lid; it < seg1 - seg0; it += wg) {
      if (join_stopped(lim)) {
        stop = true;
        break;
      }
      const uint32_t qg = indices[seg0 + it];
      const uint32_t qoff = qgoff[qg], n = qgoff[qg + 1] - qoff;
      for (uint32_t j = 0; j < n; ++j) {
        const uint32_t* r = bits + static_cast<uint64_t>(qoff + j) * Wp;
        uint32_t w[3];
#pragma unroll
        for (uint32_t k = 0; k < 3; ++k) w[k] = k < nw ? (r[i0 + k] & range_mask(i0 + k, s, e, prof)) : 0u;
        const uint64_t lo64 = static_cast<uint64_t>(w[0]) | (static_cast<uint64_t>(w[1]) << 32);
        LV(cm, j) = (lo64 >> sh) | (sh ? (static_cast<uint64_t>(w[2]) << (64u - sh)) : 0ull);
      }
      uint64_t found = 0, visited = 0;
      uint32_t top = 1;  // frames at depths 0 .. top-1
      LV(rem, 0) = LV(cm, 0);
      while (top > 0) {
        const uint32_t qn = top - 1;
        if (qn + 1 == n) {
          // the last query vertex in one step: the frame was just pushed
          uint64_t place = LV(rem, qn) & ~visited;
          if (place) {
            if (find_first) place &= 0ull - place;
            found += __popcll(place);
            if (!EXACT) {
              visited |= place & low;
              LV(map, qn) = static_cast<uint8_t>(63 - __clzll(static_cast<long long>(place)));
            }
            if (find_first) break;
          }
        } else {
          const uint64_t r = LV(rem, qn);
          if (r) {
            const uint32_t t = __ffsll(static_cast<long long>(r)) - 1;
            LV(rem, qn) = r & (r - 1);
            const uint64_t bit = 1ull << t;
            if (EXACT ? (visited & bit) : (visited & bit & low)) continue;
            // place t at depth qn and push the frame of depth qn + 1
            LV(map, qn) = static_cast<uint8_t>(t);
            visited |= EXACT ? bit : (bit & low);
            // isValidMapping for depth d = qn + 1 against mapping[0..qn]: the
            // data rows of the picks (graph-local adjacency words) must equal
            // the query's adjacency to d, bit for bit
            const uint32_t d = qn + 1;
            const uint64_t qcol = qadj[qoff + d];  // bit i: query vertices i and d adjacent
            uint64_t vm = LV(cm, d) & ~(dadj[static_cast<uint64_t>(s + t) * dAW] ^ (0ull - ((qcol >> qn) & 1ull)));
            for (uint32_t i = 0; i < qn; ++i)
              vm &= ~(dadj[static_cast<uint64_t>(s + LV(map, i)) * dAW] ^ (0ull - ((qcol >> i) & 1ull)));
            LV(rem, d) = vm;
            ++top;
            continue;
          }
        }
        // the frame at depth qn is used up
        --top;
        if (EXACT) {
          if (top) visited &= ~(1ull << LV(map, top - 1));  // the parent's pick
        } else {
          const uint32_t mq = LV(map, qn);  // mapping[qn], perhaps stale
          visited &= ~(mq < 64u ? ((1ull << mq) & low) : outside_bit);
          if (top == 1) visited = 0;
        }
        if (budget_spent(lim, steps)) {
          stop = true;
          break;
        }
      }
      if (stop) break;
      counts[seg0 + it] = found;
      my_total += found;
    }
  }
#undef LV
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

// getEdgeLabel (graph.hpp:88-93): label of the CSR entry a -> b, or 255.
__device__ __forceinline__ uint8_t csr_edge_label(uint32_t a, uint32_t b, const uint32_t* __restrict__ roff,
                                                  const uint32_t* __restrict__ col, const uint8_t* __restrict__ el) {
  for (uint32_t i = roff[a]; i < roff[a + 1]; ++i)
    if (col[i] == b) return el[i];
  return 0xFFu;
}

// joinWildcardCandidates (isomorphism.hpp:435-560) with defineMatchingOrder
// (:383-408) and the bond-label isValidMapping (:410-433).  A block is the
// reference's work-group of join_work_group_size items, one data graph at a
// time; warp w is sub-group w and takes GMCR segment slots w, w + warps, ...
// For a slot the warp picks the root (the query vertex among the first 32
// with the most candidates, highest id on ties: two warp max-reductions), and
// lane l runs one DFS per starting candidate l, l + 32, ... of the root, with
// the driver join's `visited` bitset (cleared and re-seeded with the root when
// the DFS is back at depth 1) or, for EXACT, an injective set with clean
// backtracking.  find_first ends a lane's DFS at its first match.  mapping[]
// (per query vertex) starts zeroed per lane and carries over between its DFS
// runs, as the reference's private array does.
template <bool EXACT>
__global__ void k_join_wildcard(const uint32_t* __restrict__ bits, uint64_t Wp, int prof, const uint32_t* __restrict__ qgoff,
                                const uint64_t* __restrict__ qadj, const uint32_t* __restrict__ qroff,
                                const uint32_t* __restrict__ qcol, const uint8_t* __restrict__ qel,
                                const uint32_t* __restrict__ dgoff, const uint64_t* __restrict__ dadj, uint32_t dAW,
                                const uint32_t* __restrict__ droff, const uint32_t* __restrict__ dcol,
                                const uint8_t* __restrict__ del, const uint32_t* __restrict__ offsets,
                                const uint32_t* __restrict__ indices, uint32_t G, int find_first,
                                uint64_t* __restrict__ counts, unsigned long long* __restrict__ d_total) {
  const unsigned lane = threadIdx.x & 31u, sg = threadIdx.x >> 5, nsg = blockDim.x >> 5;
  uint64_t my_total = 0;
  PairCands pc;
  uint32_t mapping[kMaxQueryNodes];
#pragma unroll 1
  for (uint32_t k = 0; k < kMaxQueryNodes; ++k) mapping[k] = 0;
  uint8_t order[kMaxQueryNodes];
  for (uint32_t g = blockIdx.x; g < G; g += gridDim.x) {
    const uint32_t s = dgoff[g], e = dgoff[g + 1], ng = e - s;
    const bool small = ng <= 64u;
    const uint32_t seg0 = offsets[g], seglen = offsets[g + 1] - seg0;
    for (uint32_t it = sg; it < seglen; it += nsg) {
      const uint32_t qg = indices[seg0 + it];
      const uint32_t qoff = qgoff[qg], n = qgoff[qg + 1] - qoff;
      if (small) pc.load(bits, Wp, qoff, n, s, e, prof);
      auto count_of = [&](uint32_t qn) -> uint32_t {
        return small ? pc.cnt[qn] : cand_count(bits + static_cast<uint64_t>(qoff + qn) * Wp, s, e, prof);
      };
      auto cand_of = [&](uint32_t qn, uint32_t idx) -> uint32_t {
        return small ? pc.at(qn, idx) : cand_at(bits + static_cast<uint64_t>(qoff + qn) * Wp, idx, s, e, prof);
      };
      // defineMatchingOrder: lane i holds query vertex i (< 32)
      const uint32_t mine = lane < n ? count_of(lane) : 0u;
      const uint32_t max_c = __reduce_max_sync(0xFFFFFFFFu, mine);
      const int root = __reduce_max_sync(0xFFFFFFFFu, (lane < n && mine == max_c) ? static_cast<int>(lane) : -1);
      order[0] = static_cast<uint8_t>(root);
#pragma unroll 1
      for (uint32_t i = 0, j = 1; i < n; ++i)
        if (static_cast<int>(i) != root) order[j++] = static_cast<uint8_t>(i);
      auto valid = [&](uint32_t cand, uint32_t depth) -> bool {
        const uint32_t qd = order[depth];
        for (uint32_t i = 0; i < depth; ++i) {
          const uint32_t qi = order[i];
          const bool qa = (qadj[qoff + qi] >> qd) & 1ull;
          if (qa != data_neighbor(mapping[qi], cand, s, ng, dadj, dAW, droff, dcol)) return false;
          if (qa && csr_edge_label(mapping[qi], cand, droff, dcol, del) != csr_edge_label(qoff + qi, qoff + qd, qroff, qcol, qel))
            return false;
        }
        return true;
      };
      uint64_t found = 0;
      for (uint32_t sc = lane; sc < max_c; sc += 32u) {
        Frame stack[kMaxQueryNodes + 2];
        uint32_t top = 0;
        const uint32_t r = order[0];
        mapping[r] = cand_of(r, sc);
        stack[top++] = {1u, 0u};
        if (!EXACT) {
          uint64_t visited = refbit(mapping[r], s);  // Bitset<uint64_t>{offset = s}
          while (top > 0) {
            const Frame fr = stack[top - 1];
            if (fr.depth == n) {
              ++found;
              --top;
              if (find_first) break;
              continue;
            }
            const uint32_t qn = order[fr.depth];
            if (fr.idx >= count_of(qn)) {
              --top;
              visited &= ~refbit(mapping[qn], s);
              if (top == 1) visited = refbit(mapping[r], s);
              continue;
            }
            const uint32_t cand = cand_of(qn, fr.idx);
            stack[top - 1].idx++;
            if (visited & refbit(cand, s)) continue;
            if (valid(cand, fr.depth)) {
              mapping[qn] = cand;
              visited |= refbit(cand, s);
              stack[top++] = {fr.depth + 1, 0u};
            }
          }
        } else {
          uint64_t used[kMaxAdjWords] = {0, 0, 0, 0};
          uint32_t placed[kMaxQueryNodes + 1];
#pragma unroll 1
          for (uint32_t k = 0; k <= n; ++k) placed[k] = 0xFFFFFFFFu;
          {
            const uint32_t t = mapping[r] - s;
            used[t >> 6] |= 1ull << (t & 63u);
          }
          while (top > 0) {
            const Frame fr = stack[top - 1];
            if (fr.depth == n) {
              ++found;
              --top;
              if (find_first) break;
              continue;
            }
            if (placed[fr.depth] != 0xFFFFFFFFu) {
              const uint32_t t = placed[fr.depth] - s;
              used[t >> 6] &= ~(1ull << (t & 63u));
              placed[fr.depth] = 0xFFFFFFFFu;
            }
            const uint32_t qn = order[fr.depth];
            if (fr.idx >= count_of(qn)) {
              --top;
              continue;
            }
            const uint32_t cand = cand_of(qn, fr.idx);
            stack[top - 1].idx++;
            const uint32_t t = cand - s;
            if ((used[t >> 6] >> (t & 63u)) & 1ull) continue;
            if (valid(cand, fr.depth)) {
              mapping[qn] = cand;
              placed[fr.depth] = cand;
              used[t >> 6] |= 1ull << (t & 63u);
              stack[top++] = {fr.depth + 1, 0u};
            }
          }
        }
      }
      my_total += found;
      uint64_t slot_total = found;
      for (int o = 16; o; o >>= 1) slot_total += __shfl_xor_sync(0xFFFFFFFFu, slot_total, o);
      if (lane == 0 && counts) counts[seg0 + it] = slot_total;
    }
  }
  for (int o = 16; o; o >>= 1) my_total += __shfl_xor_sync(0xFFFFFFFFu, my_total, o);
  if (lane == 0 && my_total) atomicAdd(d_total, static_cast<unsigned long long>(my_total));
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

// Persistent join over GMCR slots.  Each lane runs its own DFS as a flat
// state machine — one loop iteration expands one node — and pulls a new pair
// when its current one is finished, so lanes of a warp stay busy regardless of
// how uneven the pairs are.  Lanes needing work take kChunk consecutive slots
// each with one warp-aggregated atomic.
template <int AW, bool EXACT, bool FROM_PLANES>
__global__ void __launch_bounds__(128) k_join_fast(
    const uint32_t* __restrict__ bits, uint64_t Wp, const uint64_t* __restrict__ planes, uint32_t K,
    const uint32_t* __restrict__ prog_off, const uint16_t* __restrict__ prog, const uint32_t* __restrict__ cls,
    int prof, const uint32_t* __restrict__ qgoff,
    const uint8_t* __restrict__ qorder, const uint64_t* __restrict__ qsel, const uint64_t* __restrict__ qsel_id,
    const uint8_t* __restrict__ qsym, const uint32_t* __restrict__ dgoff, const uint64_t* __restrict__ dadj,
    const uint8_t* __restrict__ dsym, const uint32_t* __restrict__ indices, const uint32_t* __restrict__ pair_graph,
    const uint32_t* __restrict__ list, const unsigned long long* __restrict__ list_len, uint64_t total_slots,
    uint32_t skip_below, int find_first, uint32_t split, unsigned long long* __restrict__ cursor,
    uint64_t* __restrict__ counts, unsigned long long* __restrict__ d_total, JoinLimit lim) {
  constexpr uint32_t kChunk = 8;
  uint64_t steps = 0;
  // entries to walk (list or all slots); with split > 1 every entry is split
  // into `split` work items, item p taking the root candidates of rank = p mod
  // split, and the items' counts are merged into counts[] (zeroed beforehand)
  const uint64_t total = (list ? *list_len : total_slots) * split;
  const unsigned lane = threadIdx.x & 31u;
  uint64_t my_total = 0;
  uint64_t M[kMaxQueryNodes][AW];     // candidates of each level (graph-local)
  uint64_t cand[kMaxQueryNodes][AW];  // untried candidates of each level
  uint64_t rows[kMaxQueryNodes][AW];  // adjacency row of each level's pick
  uint32_t pick[kMaxQueryNodes];
  uint64_t next = 0, end = 0;  // this lane's claimed slot range
  uint64_t slot = 0;
  uint32_t part = 0;
  uint64_t cnt = 0;
  uint32_t n = 0, s = 0;
  const uint64_t* selp = nullptr;
  int k = -1;  // DFS level; -1 = no pair in progress
  bool have = false;
  for (;;) {
    if (k < 0) {
      if (have) {
        if (find_first && cnt) cnt = 1;
        if (split == 1) {
          counts[slot] = cnt;
          my_total += cnt;
        } else if (cnt) {
          if (!find_first) {
            atomicAdd(reinterpret_cast<unsigned long long*>(counts + slot), static_cast<unsigned long long>(cnt));
            my_total += cnt;
          } else if (atomicCAS(reinterpret_cast<unsigned long long*>(counts + slot), 0ull, 1ull) == 0ull) {
            my_total += 1;
          }
        }
        have = false;
      }
      // claim the next slot of a pair this kernel handles
      bool done = false;
      for (;;) {
        if (next >= end) {
          if (join_stopped(lim)) {
            done = true;
            break;
          }
          const unsigned am = __activemask();
          const unsigned leader = __ffs(am) - 1;
          const unsigned rank = __popc(am & ((1u << lane) - 1u));
          unsigned long long base = 0;
          if (lane == leader) base = atomicAdd(cursor, static_cast<unsigned long long>(__popc(am)) * kChunk);
          base = __shfl_sync(am, base, leader);
          next = base + static_cast<uint64_t>(rank) * kChunk;
          end = next + kChunk < total ? next + kChunk : total;
          if (next >= total) {
            done = true;
            break;
          }
        }
        const uint64_t entry = next / split;
        part = static_cast<uint32_t>(next % split);
        slot = list ? list[entry] : entry;
        ++next;
        if (pair_graph[slot] >= skip_below) break;
      }
      if (done) break;
      const uint32_t g = pair_graph[slot];
      const uint32_t qg = indices[slot];
      const uint32_t qoff = qgoff[qg];
      n = qgoff[qg + 1] - qoff;
      s = dgoff[g];
      const uint32_t e = dgoff[g + 1];
      const bool ident = !(qsym[qg] && dsym[g]);
      selp = (ident ? qsel_id : qsel) + qoff;
      for (uint32_t j = 0; j < n; ++j) {
        const uint32_t v = ident ? j : qorder[qoff + j];
        if (FROM_PLANES) mask_from_planes<AW>(planes, K, g, cls[qoff + v], prog_off, prog, M[j]);
        else extract_local<AW>(bits + static_cast<uint64_t>(qoff + v) * Wp, s, e, prof, M[j]);
      }
#pragma unroll
      for (int w = 0; w < AW; ++w) cand[0][w] = M[0][w];
      if (split > 1) {  // keep the root candidates of rank = part mod split
        uint32_t rank = 0;
#pragma unroll
        for (int w = 0; w < AW; ++w) {
          uint64_t bitsw = cand[0][w], keep = 0;
          while (bitsw) {
            const uint64_t low = bitsw & (0ull - bitsw);
            if (rank % split == part) keep |= low;
            ++rank;
            bitsw ^= low;
          }
          cand[0][w] = keep;
        }
      }
      cnt = 0;
      k = 0;
      have = true;
      continue;
    }
    // one DFS node at level k
    bool empty = true;
#pragma unroll
    for (int w = 0; w < AW; ++w) empty &= cand[k][w] == 0;
    if (empty) {
      --k;
      if (budget_spent(lim, steps)) break;
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
      const uint64_t keep_set = 0ull - ((sl >> i) & 1ull);  // all ones when adjacent in the query
#pragma unroll
      for (int w = 0; w < AW; ++w) nx[w] &= ~(rows[i][w] ^ keep_set) ;
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
      if (find_first && cnt) k = -1;
      continue;
    }
    ++k;
#pragma unroll
    for (int w = 0; w < AW; ++w) cand[k][w] = nx[w];
  }
  for (int o = 16; o; o >>= 1) my_total += __shfl_xor_sync(0xFFFFFFFFu, my_total, o);
  if (lane == 0 && my_total) atomicAdd(d_total, static_cast<unsigned long long>(my_total));
}

// Two-phase join for pairs whose query has <= kPhaseLevels vertices.
// Phase A (k_pair_masks): per slot of a chunk and per level j, the candidate
// set of the query vertex placed at level j = AND of its class's plane program
// for the slot's data graph, stored [slot-in-chunk][level] (coalesced: one
// 128-byte line per slot, so a pair's later levels hit in cache).
// Phase B (k_join_masks): the DFS as a flat per-lane state machine whose pair
// setup is just the load of those masks (issued one pair ahead, so the DRAM
// latency of a refill overlaps the current pair's DFS), with the per-level
// state in shared memory ([level][thread]).  Trying a candidate t at level k is O(1):
// next = base[k+1] & (row(t) or ~row(t)) [& ~used]; base[k+2] is computed
// once per descent.
constexpr uint32_t kPhaseLevels = 16;
constexpr uint32_t kPhaseThreads = 256;

// Work layout: a warp takes 32 consecutive slots per round, one lane per slot
// for the slot's metadata and setup record, then the round's sum of query
// sizes (slot, level) items with every lane busy; an item finds its slot by a
// binary search over the lanes' exclusive prefix sums (warp shuffles).
__global__ void __launch_bounds__(256) k_pair_masks(
    const uint64_t* __restrict__ planes, uint32_t K, uint32_t AW, const uint32_t* __restrict__ prog_off,
    const uint16_t* __restrict__ prog,
    const uint32_t* __restrict__ cls, const uint32_t* __restrict__ qgoff, const uint8_t* __restrict__ qorder,
    const uint8_t* __restrict__ qsym, const uint32_t* __restrict__ dgoff, const uint8_t* __restrict__ dsym,
    const uint32_t* __restrict__ indices, const uint32_t* __restrict__ pair_graph, uint64_t slot0, uint64_t count,
    uint64_t* __restrict__ masks, uint4* __restrict__ rec, uint32_t skip_below, uint32_t* __restrict__ overflow,
    unsigned long long* __restrict__ overflow_len, uint64_t* __restrict__ counts) {
  const unsigned lane = threadIdx.x & 31u;
  const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
  for (uint64_t s0 = warp * 32; s0 < count; s0 += nwarps * 32) {
    const uint64_t local = s0 + lane;
    uint32_t n = 0, qoff = 0, g = 0, items = 0;
    bool ident = true;
    if (local < count) {
      const uint64_t slot = slot0 + local;
      const uint32_t qg = indices[slot];
      qoff = qgoff[qg];
      n = qgoff[qg + 1] - qoff;
      g = pair_graph[slot];
      ident = !(qsym[qg] && dsym[g]);
      const uint32_t ds = dgoff[g];
      // queries over kPhaseLevels vertices and molecules over 64 atoms (a
      // vertex set wider than one word) go to the generic kernel
      const bool generic = n > kPhaseLevels || dgoff[g + 1] - ds > 64u;
      // the pair's setup record: first data vertex, query size | flags, query offset, data graph
      rec[local] = make_uint4(ds, n | (ident ? 0x100u : 0u) | (generic ? 0x200u : 0u), qoff, g);
      if (generic && g >= skip_below) {  // joined by the generic kernel, which accumulates into counts
        overflow[atomicAdd(overflow_len, 1ull)] = static_cast<uint32_t>(slot);
        counts[slot] = 0;
      }
      items = generic ? 0u : n;
    }
    uint32_t incl = items;
#pragma unroll
    for (unsigned o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += v;
    }
    const uint32_t excl = incl - items;
    const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    for (uint32_t base = 0; base < total; base += 32) {
      const uint32_t it = base + lane;
      // owner: the last lane whose exclusive prefix is <= it
      uint32_t pos = 0;
#pragma unroll
      for (uint32_t step = 16; step; step >>= 1) {
        const uint32_t cand = pos + step;
        const uint32_t e = __shfl_sync(0xFFFFFFFFu, excl, cand & 31u);
        if (cand < 32u && e <= it) pos = cand;
      }
      const uint32_t o_excl = __shfl_sync(0xFFFFFFFFu, excl, pos);
      const uint32_t o_qoff = __shfl_sync(0xFFFFFFFFu, qoff, pos);
      const uint32_t o_g = __shfl_sync(0xFFFFFFFFu, g, pos);
      const bool o_ident = __shfl_sync(0xFFFFFFFFu, static_cast<unsigned>(ident), pos) != 0u;
      if (it >= total) continue;
      const uint32_t j = it - o_excl;
      const uint32_t c = cls[o_qoff + (o_ident ? j : qorder[o_qoff + j])];
      // word 0 of each plane: the graph's vertex set fits one word
      const uint64_t* pb = planes + static_cast<uint64_t>(o_g >> 5) * K * AW * 32 + (o_g & 31u);
      uint64_t m = ~0ull;
      const uint32_t e1 = prog_off[c + 1];
      for (uint32_t e = prog_off[c]; e < e1; ++e) m &= pb[static_cast<uint64_t>(prog[e]) * AW * 32];
      masks[(s0 + pos) * kPhaseLevels + j] = m;
    }
  }
}

// DAW: words per adjacency row of the data batch (the pairs here use word 0).
template <bool EXACT, uint32_t DAW>
__global__ void __launch_bounds__(kPhaseThreads) k_join_masks(
    const uint64_t* __restrict__ masks, const uint4* __restrict__ rec, uint64_t slot0, uint64_t count,
    const uint64_t* __restrict__ qsel, const uint64_t* __restrict__ qsel_id, const uint64_t* __restrict__ dadj,
    uint32_t skip_below, int find_first, uint32_t kChunk, unsigned long long* __restrict__ cursor,
    uint64_t* __restrict__ counts, unsigned long long* __restrict__ d_total, JoinLimit lim) {
  extern __shared__ uint64_t sm[];
  uint64_t steps = 0;
  const unsigned tid = threadIdx.x, lane = tid & 31u;
  uint64_t* cand = sm;
  uint64_t* base = sm + kPhaseLevels * kPhaseThreads;
  uint8_t* pk = reinterpret_cast<uint8_t*>(sm + 2 * kPhaseLevels * kPhaseThreads);
#define AT(arr, lvl) arr[(lvl) * kPhaseThreads + tid]
  uint64_t my_total = 0;
  uint64_t next = 0, end = 0, local = 0, cnt = 0;
  uint32_t n = 0, s = 0;
  const uint64_t* selp = nullptr;
  uint64_t used = 0;
  int k = -1;
  bool have = false;
  // the next slot's record and first two level masks, loaded one pair ahead
  uint4 pr = make_uint4(0, 0, 0, 0);
  uint64_t pm0 = 0, pm1 = 0, plocal = 0;
  bool pre = false;
  auto fetch = [&]() {
    pre = false;
    if (next >= end) {
      if (join_stopped(lim)) return;
      const unsigned am = __activemask();
      const unsigned leader = __ffs(am) - 1;
      const unsigned rank = __popc(am & ((1u << lane) - 1u));
      unsigned long long b = 0;
      if (lane == leader) b = atomicAdd(cursor, static_cast<unsigned long long>(__popc(am)) * kChunk);
      b = __shfl_sync(am, b, leader);
      next = b + static_cast<uint64_t>(rank) * kChunk;
      end = next + kChunk < count ? next + kChunk : count;
      if (next >= count) return;
    }
    plocal = next++;
    pr = rec[plocal];
    pm0 = masks[plocal * kPhaseLevels];
    pm1 = masks[plocal * kPhaseLevels + 1];
    pre = true;
  };
  fetch();
  for (;;) {
    if (k < 0) {
      if (have) {
        if (find_first && cnt) cnt = 1;
        counts[slot0 + local] = cnt;
        my_total += cnt;
        have = false;
      }
      if (!pre) break;
      local = plocal;
      const uint4 r = pr;  // first data vertex, query size | order flag, query offset, data graph
      const uint64_t m0 = pm0, m1 = pm1;
      fetch();
      if (r.w < skip_below) continue;
      n = r.y & 0xFFu;
      if (r.y & 0x200u) continue;  // in the overflow list (generic kernel)
      s = r.x;
      selp = ((r.y & 0x100u) ? qsel_id : qsel) + r.z;
      AT(cand, 0) = m0;
      AT(base, 1) = m1;
      used = 0;
      cnt = 0;
      k = 0;
      have = true;
      continue;
    }
    const uint64_t ck = AT(cand, k);
    if (!ck) {
      --k;
      if (EXACT && k >= 0) used &= ~(1ull << AT(pk, k));
      if (budget_spent(lim, steps)) break;
      continue;
    }
    const uint32_t t = __ffsll(static_cast<long long>(ck)) - 1;
    AT(cand, k) = ck & (ck - 1);
    const uint64_t rw = dadj[static_cast<uint64_t>(s + t) * DAW];
    const uint64_t keep = 0ull - ((selp[k + 1] >> k) & 1ull);
    uint64_t nx = AT(base, k + 1) & ~(rw ^ keep);
    if (EXACT) nx &= ~(used | (1ull << t));
    if (static_cast<uint32_t>(k + 1) == n - 1) {
      cnt += __popcll(nx);
      if (find_first && cnt) k = -1;
      continue;
    }
    if (!nx) continue;
    AT(pk, k) = static_cast<uint8_t>(t);
    if (EXACT) used |= 1ull << t;
    AT(cand, k + 1) = nx;
    const uint64_t sl2 = selp[k + 2];
    uint64_t b2 = masks[local * kPhaseLevels + k + 2] & ~(rw ^ (0ull - ((sl2 >> k) & 1ull)));
    for (int i = 0; i < k; ++i) b2 &= ~(dadj[static_cast<uint64_t>(s + AT(pk, i)) * DAW] ^ (0ull - ((sl2 >> i) & 1ull)));
    AT(base, k + 2) = b2;
    ++k;
  }
#undef AT
  for (int o = 16; o; o >>= 1) my_total += __shfl_xor_sync(0xFFFFFFFFu, my_total, o);
  if (lane == 0 && my_total) atomicAdd(d_total, static_cast<unsigned long long>(my_total));
}

// Join phase B, default form (sigmo_tuning.join_kernel = 2): the per-lane DFS
// machine of k_join_masks with 9 bytes of shared state per level and lane,
// base[j] (level j's candidates under the constraints of levels 0..j-2) and
// pk[j] (level j's current pick).  The untried candidates of the current level
// live in a register; a backtrack to level k recomputes them as base[k] AND
// the constraint of pick[k-1]'s row, above pick[k].  Four 256-thread CTAs fit
// on an SM.  A descent whose level-(k+2) base mask comes out empty is dropped:
// every candidate of level k+1 would then extend to nothing, so the subtree
// counts 0.  Work: each CTA first takes slots from its own contiguous region
// of the chunk, so its lanes join neighbouring molecules whose adjacency rows
// stay in L1 (measured: L1 hit rate 82 % against 33 % with one global work
// cursor), then from a tail pool shared by all CTAs (pool16 sixteenths of the
// chunk) that evens out the CTAs' finishing times.
constexpr size_t kLaneBytesPerThread = kPhaseLevels * (8 + 1);

template <bool EXACT, uint32_t DAW>
__global__ void __launch_bounds__(kPhaseThreads, 4) k_join_lanes(
    const uint64_t* __restrict__ masks, const uint4* __restrict__ rec, uint64_t slot0, uint64_t count,
    const uint64_t* __restrict__ qsel, const uint64_t* __restrict__ qsel_id, const uint64_t* __restrict__ dadj,
    uint32_t skip_below, int find_first, uint32_t pool16, unsigned long long* __restrict__ cursor,
    uint64_t* __restrict__ counts, unsigned long long* __restrict__ d_total, JoinLimit lim) {
  extern __shared__ uint64_t sm[];
  __shared__ unsigned long long s_taken;  // slots of this CTA's region handed out so far
  const unsigned tid = threadIdx.x, lane = tid & 31u;
  uint64_t* base = sm;
  uint8_t* pk = reinterpret_cast<uint8_t*>(sm + kPhaseLevels * kPhaseThreads);
#define AT(arr, lvl) arr[(lvl) * kPhaseThreads + tid]
  const uint64_t shared_slots = count / 16u * (pool16 < 16u ? pool16 : 16u);
  const uint64_t rlen = (count - shared_slots) / gridDim.x;
  const uint64_t pool0 = rlen * gridDim.x;
  const uint64_t r0 = static_cast<uint64_t>(blockIdx.x) * rlen;
  if (tid == 0) s_taken = 0;
  __syncthreads();
  uint64_t steps = 0, my_total = 0, local = 0, cnt = 0, used = 0, rem = 0;
  uint32_t n = 0, s = 0;
  const uint64_t* selp = qsel;
  int k = -1;
  bool have = false;
  // the next slot's record and first two level masks, loaded one pair ahead
  uint4 pr = make_uint4(0, 0, 0, 0);
  uint64_t pm0 = 0, pm1 = 0, plocal = 0;
  bool pre = false;
  auto fetch = [&]() {
    pre = false;
    if (join_stopped(lim)) return;
    const unsigned am = __activemask();
    const unsigned leader = __ffs(am) - 1, c = __popc(am);
    const unsigned rank = __popc(am & ((1u << lane) - 1u));
    unsigned long long rb = 0, pb = 0;
    if (lane == leader) {
      rb = atomicAdd(&s_taken, static_cast<unsigned long long>(c));
      const uint64_t in_region = rb < rlen ? (rlen - rb < c ? rlen - rb : c) : 0ull;
      if (c > in_region) pb = atomicAdd(cursor, static_cast<unsigned long long>(c - in_region));
    }
    rb = __shfl_sync(am, rb, leader);
    pb = __shfl_sync(am, pb, leader);
    const uint64_t in_region = rb < rlen ? (rlen - rb < c ? rlen - rb : c) : 0ull;
    const uint64_t slot = rank < in_region ? r0 + rb + rank : pool0 + pb + (rank - in_region);
    if (slot >= count) return;
    plocal = slot;
    pr = rec[slot];
    pm0 = masks[slot * kPhaseLevels];
    pm1 = masks[slot * kPhaseLevels + 1];
    pre = true;
  };
  fetch();
  for (;;) {
    if (k < 0) {
      if (have) {
        if (find_first && cnt) cnt = 1;
        counts[slot0 + local] = cnt;
        my_total += cnt;
        have = false;
      }
      if (!pre) break;
      local = plocal;
      const uint4 r = pr;  // first data vertex, query size | flags, query offset, data graph
      const uint64_t m0 = pm0, m1 = pm1;
      fetch();
      if (r.w < skip_below || (r.y & 0x200u)) continue;  // literal join, or the overflow list (generic kernel)
      n = r.y & 0xFFu;
      s = r.x;
      selp = ((r.y & 0x100u) ? qsel_id : qsel) + r.z;
      AT(base, 0) = m0;
      AT(base, 1) = m1;
      rem = m0;
      used = 0;
      cnt = 0;
      k = 0;
      have = true;
      continue;
    }
    if (!rem) {  // back to level k-1: its untried candidates from its base and its parent's row
      if (budget_spent(lim, steps)) break;
      if (k == 0) {
        k = -1;
        continue;
      }
      --k;
      const uint32_t p = AT(pk, k);
      if (EXACT) used &= ~(1ull << p);
      uint64_t f = AT(base, k);
      if (k > 0) {
        const uint64_t rw = dadj[static_cast<uint64_t>(s + AT(pk, k - 1)) * DAW];
        f &= ~(rw ^ (0ull - ((static_cast<uint32_t>(selp[k]) >> (k - 1)) & 1u)));
        if (EXACT) f &= ~used;
      }
      rem = f & ~((2ull << p) - 1ull);
      continue;
    }
    const uint32_t t = __ffsll(static_cast<long long>(rem)) - 1;
    rem &= rem - 1;
    const uint64_t rw = dadj[static_cast<uint64_t>(s + t) * DAW];
    uint64_t nx = AT(base, k + 1) & ~(rw ^ (0ull - ((static_cast<uint32_t>(selp[k + 1]) >> k) & 1u)));
    if (EXACT) nx &= ~(used | (1ull << t));
    if (static_cast<uint32_t>(k + 2) >= n) {
      cnt += __popcll(nx);
      if (find_first && cnt) k = -1;
      continue;
    }
    if (!nx) continue;
    const uint32_t sl2 = static_cast<uint32_t>(selp[k + 2]);
    uint64_t b2 = masks[local * kPhaseLevels + k + 2] & ~(rw ^ (0ull - ((sl2 >> k) & 1u)));
    for (int i = 0; i < k && b2; ++i) b2 &= ~(dadj[static_cast<uint64_t>(s + AT(pk, i)) * DAW] ^ (0ull - ((sl2 >> i) & 1u)));
    if (!b2) continue;  // level k+2 would be empty below every candidate of level k+1
    AT(pk, k) = static_cast<uint8_t>(t);
    if (EXACT) used |= 1ull << t;
    AT(base, k + 2) = b2;
    ++k;
    rem = nx;
  }
#undef AT
  for (int o = 16; o; o >>= 1) my_total += __shfl_xor_sync(0xFFFFFFFFu, my_total, o);
  if (lane == 0 && my_total) atomicAdd(d_total, static_cast<unsigned long long>(my_total));
}

// Position of the r-th (0-based) set bit of m; m has more than r set bits.
__device__ __forceinline__ uint32_t nth_set32(uint32_t m, uint32_t r) {
  uint32_t pos = 0, c = __popc(m & 0xFFFFu);
  if (r >= c) { r -= c; pos += 16; m >>= 16; }
  c = __popc(m & 0xFFu);
  if (r >= c) { r -= c; pos += 8; m >>= 8; }
  c = __popc(m & 0xFu);
  if (r >= c) { r -= c; pos += 4; m >>= 4; }
  c = __popc(m & 0x3u);
  if (r >= c) { r -= c; pos += 2; m >>= 2; }
  if (r >= (m & 1u)) pos += 1;
  return pos;
}
__device__ __forceinline__ uint32_t nth_set64(uint64_t m, uint32_t r) {
  const uint32_t lo = static_cast<uint32_t>(m), c = __popc(lo);
  const bool up = r >= c;
  return (up ? 32u : 0u) + nth_set32(up ? static_cast<uint32_t>(m >> 32) : lo, up ? r - c : r);
}

// Phase B, warp-cooperative form (k_join_frontier).  A warp keeps up to 32
// pairs in flight (slot p: its root candidates, count and live-entry count).
// A partial embedding of depth L >= 1 is an entry {candidates left at level
// L; meta = pair | vertex placed at level L-1 << 5 | parent entry << 11} in a
// per-warp pool where each level's entries form one region, stacked in level
// order.  A round takes the next 32 (entry, candidate) items of the current
// level L, one per lane: the lane rebuilds the level-(L+1) constraint by
// walking the parent chain, tries its candidate (the same test as the
// per-lane machine) and appends the child entry at level L+1, or adds the
// popcount when L+1 is the last level.  The warp goes one level deeper once
// the next level holds a full round (levels above kFrontDeep: any entry), and
// back up when the current level is used up, so a level holds at most 63
// entries (31 above kFrontDeep) and the pool is bounded by kFrontPool.
// Counts are order-independent sums, so they equal the per-lane machine's.
constexpr uint32_t kFrontPairs = 32;
constexpr uint32_t kFrontDeep = 4;
constexpr uint32_t kFrontPool = kFrontDeep * 63u + (kPhaseLevels - 2u - kFrontDeep) * 32u;
constexpr uint32_t kFrontWarps = 8;
constexpr uint32_t kFrontFree = 0xFFFFFFFFu;
struct FrontWarp {
  unsigned long long pcnt[kFrontPairs];  // embeddings found per pair slot
  uint64_t pcand[kFrontPairs];           // level-0 candidates not yet taken
  uint64_t ecand[kFrontPool];
  uint32_t emeta[kFrontPool];
  // per pair slot: first data vertex of the graph, query offset | identity-order
  // flag << 31, chunk-local slot (kFrontFree when the slot is free), query size
  uint4 pinfo[kFrontPairs];
  uint32_t pref[kFrontPairs];  // live entries (root included)
  uint16_t head[kPhaseLevels + 1], tail[kPhaseLevels + 1];
};

template <bool EXACT, uint32_t DAW>
__global__ void __launch_bounds__(kFrontWarps * 32, 3) k_join_frontier(
    const uint64_t* __restrict__ masks, const uint4* __restrict__ rec, uint64_t slot0, uint64_t count,
    const uint64_t* __restrict__ qsel, const uint64_t* __restrict__ qsel_id, const uint64_t* __restrict__ dadj,
    uint32_t skip_below, int find_first, uint32_t kChunk, unsigned long long* __restrict__ cursor,
    uint64_t* __restrict__ counts, unsigned long long* __restrict__ d_total, JoinLimit lim) {
  extern __shared__ __align__(16) unsigned char front_raw[];
  uint64_t rounds = 0;
  FrontWarp& w = reinterpret_cast<FrontWarp*>(front_raw)[threadIdx.x >> 5];
  const unsigned lane = threadIdx.x & 31u, lt = (1u << lane) - 1u;
  constexpr unsigned kAll = 0xFFFFFFFFu;
  w.pinfo[lane].z = kFrontFree;
  w.pcand[lane] = 0;
  w.pref[lane] = 0;
  if (lane <= kPhaseLevels) w.head[lane] = w.tail[lane] = 0;
  __syncwarp();
  uint64_t next = 0, end = 0;  // warp-uniform range of chunk-local slots
  bool more = true;
  uint64_t my_total = 0;
  uint32_t L = 0;
  for (;;) {
    // the budget counts this warp's rounds (warp-uniform)
    if (lim.budget && ++rounds > lim.budget) {
      if (lane == 0) atomicOr(lim.status, kJoinStatusBudget);
      break;
    }
    if (L == 0 && more) {
      // fill the free pair slots (lane i owns slot i) from the work range
      bool fr = w.pinfo[lane].z == kFrontFree;
      unsigned F = __ballot_sync(kAll, fr);
      while (F && more) {
        if (next >= end) {
          if (__shfl_sync(kAll, join_stopped(lim) ? 1u : 0u, 0)) {
            more = false;
            break;
          }
          unsigned long long b = 0;
          if (lane == 0) b = atomicAdd(cursor, 32ull * kChunk);
          b = __shfl_sync(kAll, b, 0);
          next = b;
          end = b + 32ull * kChunk < count ? b + 32ull * kChunk : count;
          if (next >= count) {
            more = false;
            break;
          }
        }
        const uint32_t avail = static_cast<uint32_t>(end - next < 32 ? end - next : 32);
        const uint32_t take = min(static_cast<uint32_t>(__popc(F)), avail);
        const uint32_t rank = __popc(F & lt);
        if (fr && rank < take) {
          const uint64_t local = next + rank;
          const uint4 r = rec[local];  // first data vertex, query size | flags, query offset, data graph
          if (r.w >= skip_below && !(r.y & 0x200u)) {
            const uint64_t c0 = masks[local * kPhaseLevels];
            if (c0) {
              w.pinfo[lane] = make_uint4(r.x, r.z | ((r.y & 0x100u) ? 0x80000000u : 0u), static_cast<uint32_t>(local), r.y & 0xFFu);
              w.pcand[lane] = c0;
              w.pcnt[lane] = 0;
              w.pref[lane] = 1;
              fr = false;
            } else {
              counts[slot0 + local] = 0;  // no candidate for the first query vertex
            }
          }
        }
        next += take;
        F = __ballot_sync(kAll, fr);
      }
      __syncwarp();
    }
    // ---- one round at level L: this lane's source entry (L = 0: pair slot)
    const uint32_t head = w.head[L], tail = w.tail[L];
    uint64_t cand;
    if (L == 0) cand = w.pcand[lane];
    else cand = head + lane < tail ? w.ecand[head + lane] : 0ull;
    const uint32_t c = __popcll(cand);
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kAll, incl, o);
      if (lane >= static_cast<unsigned>(o)) incl += y;
    }
    const uint32_t excl = incl - c;
    const uint32_t total = __shfl_sync(kAll, incl, 31);
    if (total) {
      const uint32_t nitems = total < 32u ? total : 32u;
      // the owner of item `lane`: the first source lane whose inclusive
      // count exceeds it (binary search over the non-decreasing counts)
      uint32_t o = 0;
#pragma unroll
      for (uint32_t step = 16; step; step >>= 1) {
        const uint32_t v = __shfl_sync(kAll, incl, o + step - 1u);
        if (v <= lane) o += step;
      }
      o = o < 31u ? o : 31u;
      const uint32_t oexcl = __shfl_sync(kAll, excl, o), oincl = __shfl_sync(kAll, incl, o);
      const uint64_t ocand = __shfl_sync(kAll, cand, o);
      const bool item = lane < nitems;
      bool child = false, exhausted = false;
      uint64_t nx = 0;
      uint32_t p = 0, t = 0;
      if (item) {
        t = nth_set64(ocand, lane - oexcl);
        const bool last_of_owner = lane + 1u == (oincl < nitems ? oincl : nitems);
        uint32_t meta = 0;
        if (L == 0) {
          p = o;
        } else {
          meta = w.emeta[head + o];
          p = meta & 31u;
        }
        if (last_of_owner) {  // the owner's candidates up to t are taken
          const uint64_t left = ocand & ~((2ull << t) - 1ull);
          if (L == 0) w.pcand[o] = left;
          else w.ecand[head + o] = left;
          exhausted = left == 0;
        }
        const uint4 pi = w.pinfo[p];
        const uint32_t s = pi.x, sv = pi.y, local = pi.z, n = pi.w;
        const uint64_t* selp = ((sv >> 31) ? qsel_id : qsel) + (sv & 0x7FFFFFFFu);
        const uint64_t sl = selp[L + 1];
        uint64_t b = masks[static_cast<uint64_t>(local) * kPhaseLevels + L + 1u];
        uint64_t used = 0;
        if (L) {  // constraints of the vertices placed at levels L-1 .. 0
          uint32_t m = meta;
          for (int i = static_cast<int>(L) - 1;; --i) {
            const uint32_t ti = (m >> 5) & 63u;
            b &= ~(dadj[static_cast<uint64_t>(s + ti) * DAW] ^ (0ull - ((sl >> i) & 1ull)));
            if (EXACT) used |= 1ull << ti;
            if (i == 0) break;
            m = w.emeta[m >> 11];
          }
        }
        const uint64_t rw = dadj[static_cast<uint64_t>(s + t) * DAW];
        nx = b & ~(rw ^ (0ull - ((sl >> L) & 1ull)));
        if (EXACT) nx &= ~(used | (1ull << t));
        if (!(find_first && w.pcnt[p])) {
          if (L + 1u == n - 1u) {
            if (nx) atomicAdd(&w.pcnt[p], static_cast<unsigned long long>(__popcll(nx)));
          } else {
            child = nx != 0;
          }
        }
      }
      // children at level L + 1, in lane order
      const unsigned cb = __ballot_sync(kAll, child);
      const uint32_t at = w.tail[L + 1];
      if (child) {
        const uint32_t pos = at + __popc(cb & lt);
        if (pos < kFrontPool) {  // always true: the level bounds above sum to kFrontPool
          w.ecand[pos] = nx;
          w.emeta[pos] = p | (t << 5) | ((L ? head + o : 0u) << 11);
          atomicAdd(&w.pref[p], 1u);
        }
      }
      __syncwarp();
      if (lane == 0 && cb) {
        const uint32_t nt = min(at + static_cast<uint32_t>(__popc(cb)), kFrontPool);
        w.tail[L + 1] = static_cast<uint16_t>(nt);
        w.head[L + 2] = w.tail[L + 2] = static_cast<uint16_t>(nt);  // level L+2 is empty
      }
      // entries used up in this round release their pair; the last one ends it
      if (exhausted && atomicSub(&w.pref[p], 1u) == 1u) {
        unsigned long long cn = w.pcnt[p];
        if (find_first && cn) cn = 1;
        counts[slot0 + w.pinfo[p].z] = cn;
        my_total += cn;
        w.pinfo[p].z = kFrontFree;
      }
      if (L) {  // the used-up entries are a prefix of the level
        const unsigned gone = __ballot_sync(kAll, incl <= 32u);
        const uint32_t lead = gone == kAll ? 32u : static_cast<uint32_t>(__ffs(~gone) - 1);
        if (lane == 0) w.head[L] = static_cast<uint16_t>(head + lead < tail ? head + lead : tail);
      }
      __syncwarp();
    }
    // ---- next level (warp-uniform)
    const bool left = L ? w.head[L] < w.tail[L] : __any_sync(kAll, w.pcand[lane] != 0);
    const uint32_t waiting = w.tail[L + 1] - w.head[L + 1];
    const uint32_t thr = L + 1u <= kFrontDeep ? 32u : 1u;
    if (waiting && (waiting >= thr || !left)) {
      ++L;
      continue;
    }
    if (!left) {
      if (L) {
        const uint16_t start = L == 1 ? 0 : w.tail[L - 1];
        __syncwarp();
        if (lane == 0) w.head[L] = w.tail[L] = w.head[L + 1] = w.tail[L + 1] = start;
        __syncwarp();
        --L;
      } else if (!more) {
        break;  // no pair in flight and no work left
      }
    }
  }
  for (int o = 16; o; o >>= 1) my_total += __shfl_xor_sync(0xFFFFFFFFu, my_total, o);
  if (lane == 0 && my_total) atomicAdd(d_total, static_cast<unsigned long long>(my_total));
}

}  // namespace

int launch_join_literal(Queue* q, const Graph* query, const Graph* data, const Candidates* c, Gmcr* m, int find_first,
                        uint32_t graph_begin, uint32_t graph_end, uint64_t* d_total, uint32_t q_begin, uint32_t q_end) {
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
  // the common case (graphs of <= 64 vertices, queries of <= kLitLevels) keeps
  // its per-level state in shared memory
  uint32_t range_max = data->max_nodes;
  if (range_max > 64u) {
    range_max = 0;
    for (uint32_t g = graph_begin; g < graph_end; ++g)
      range_max = std::max(range_max, data->host_graph_offsets[g + 1] - data->host_graph_offsets[g]);
  }
  if (range_max <= 64u && query->max_nodes <= kLitLevels && wg <= 256u) {
    const size_t smem = kLitBytesPerThread * wg;
    auto kern = exact ? k_join_literal_small<true> : k_join_literal_small<false>;
    SIGMO_TRY(allow_max_dynamic_smem(reinterpret_cast<const void*>(kern), q->device));
    kern<<<grid, wg, smem, q->stream>>>(c->bits, c->Wp, q->opts.profile, query->graph_offsets, query->adj,
                                        data->graph_offsets, data->adj, data->adj_words, m->offsets, m->indices, graph_begin,
                                        graph_end, q_begin, q_end, find_first, m->counts, tot, join_limit(q));
    return check_launch(q, "k_join_literal_small");
  }
  if (exact)
    k_join_literal<true><<<grid, wg, 0, q->stream>>>(c->bits, c->Wp, q->opts.profile, query->graph_offsets, query->adj,
                                                      data->graph_offsets, data->adj, data->adj_words, data->row_offsets,
                                                      data->column_indices, m->offsets, m->indices, graph_begin, graph_end,
                                                      q_begin, q_end, find_first, m->counts, tot, join_limit(q));
  else
    k_join_literal<false><<<grid, wg, 0, q->stream>>>(c->bits, c->Wp, q->opts.profile, query->graph_offsets, query->adj,
                                                       data->graph_offsets, data->adj, data->adj_words, data->row_offsets,
                                                       data->column_indices, m->offsets, m->indices, graph_begin, graph_end,
                                                       q_begin, q_end, find_first, m->counts, tot, join_limit(q));
  return check_launch(q, "k_join_literal");
}

int launch_join_wildcard(Queue* q, const Graph* query, const Graph* data, const Candidates* c, Gmcr* m, int find_first,
                         uint64_t* d_total) {
  if (query->max_nodes > kMaxQueryNodes)
    return fail(SIGMO_ERR_DOMAIN, "query graphs of up to %u vertices are supported (largest: %u)", kMaxQueryNodes, query->max_nodes);
  const bool exact = q->opts.profile == kProfileExact;
  if (exact && data->max_nodes > 64u * kMaxAdjWords)
    return fail(SIGMO_ERR_DOMAIN, "exact profile supports data graphs of at most %u vertices", 64u * kMaxAdjWords);
  const uint32_t wg = q->opts.join_work_group_size ? q->opts.join_work_group_size : 128u;
  if (wg > 1024u || (wg & 31u)) return fail(SIGMO_ERR_INVALID, "join work-group size %u must be a multiple of 32 <= 1024", wg);
  const uint32_t G = data->num_graphs;
  if (!G) return SIGMO_OK;
  const unsigned grid = std::min<uint32_t>(G, 148u * 64u);
  auto* tot = reinterpret_cast<unsigned long long*>(d_total);
  if (exact)
    k_join_wildcard<true><<<grid, wg, 0, q->stream>>>(c->bits, c->Wp, q->opts.profile, query->graph_offsets, query->adj,
                                                      query->row_offsets, query->column_indices, query->edge_labels,
                                                      data->graph_offsets, data->adj, data->adj_words, data->row_offsets,
                                                      data->column_indices, data->edge_labels, m->offsets, m->indices, G,
                                                      find_first, m->counts, tot);
  else
    k_join_wildcard<false><<<grid, wg, 0, q->stream>>>(c->bits, c->Wp, q->opts.profile, query->graph_offsets, query->adj,
                                                       query->row_offsets, query->column_indices, query->edge_labels,
                                                       data->graph_offsets, data->adj, data->adj_words, data->row_offsets,
                                                       data->column_indices, data->edge_labels, m->offsets, m->indices, G,
                                                       find_first, m->counts, tot);
  return check_launch(q, "k_join_wildcard");
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
                                                       data->adj, data->sym, m->indices, m->pair_graph, nullptr, nullptr, \
                                                       m->total, skip, find_first, 1u, cursor, m->counts, tot, \
                                                       join_limit(q))
  switch (data->adj_words) {
    case 1: if (exact) SIGMO_JOIN_FAST(1, true); else SIGMO_JOIN_FAST(1, false); break;
    case 2: if (exact) SIGMO_JOIN_FAST(2, true); else SIGMO_JOIN_FAST(2, false); break;
    default: if (exact) SIGMO_JOIN_FAST(4, true); else SIGMO_JOIN_FAST(4, false); break;
  }
#undef SIGMO_JOIN_FAST
  return check_launch(q, "k_join_fast");
}

int launch_join_fast_planes(Queue* q, const Graph* query, const Graph* data, const PlaneProgram& pp, const uint64_t* planes,
                            uint32_t planes_rows, const uint16_t* prog, Gmcr* m, int find_first, uint64_t* d_total,
                            uint32_t reserve) {
  if (!m->total) return SIGMO_OK;
  if (query->max_nodes > kMaxQueryNodes)
    return fail(SIGMO_ERR_DOMAIN, "query graphs of up to %u vertices are supported (largest: %u)", kMaxQueryNodes, query->max_nodes);
  const bool exact = q->opts.profile == kProfileExact;
  SIGMO_TRY(launch_query_order(const_cast<Graph*>(query)));
  const uint32_t skip = exact ? 0u : data->low_offset_graphs;
  void* buf = nullptr;
  SIGMO_TRY(tmp_alloc(q, &buf, 256 + 4ull * m->total));
  // [0] work cursor of the even chunks, [1] generic-join cursor, [2] overflow length, [3] odd chunks' cursor
  auto* ctr = static_cast<unsigned long long*>(buf);
  uint32_t* overflow = reinterpret_cast<uint32_t*>(static_cast<char*>(buf) + 256);
  SIGMO_CUDA_TRY(cudaMemsetAsync(ctr, 0, 256, q->stream));
  auto* tot = reinterpret_cast<unsigned long long*>(d_total);
  // two-phase join, in chunks of slots, for the pairs of queries of <= 16
  // vertices and molecules of <= 64 atoms; the rest go to the overflow list
  int rc = SIGMO_OK;
  bool two = false;
  {
    const sigmo_tuning& tn = q->tune;
    const uint64_t chunk = std::min<uint64_t>(m->total, static_cast<uint64_t>(tn.mask_chunk_slots) << 20);
    // several chunks: even ones on the main stream, odd ones on the aux
    // stream, each stream with its own mask buffer and work cursor, so one
    // chunk's level masks run beside the previous chunk's persistent join
    two = m->total > chunk;
    const size_t mbytes = 8ull * kPhaseLevels * chunk + 16ull * chunk;
    void* mbuf[2] = {nullptr, nullptr};
    rc = tmp_alloc(q, &mbuf[0], mbytes);
    if (!rc && two) rc = tmp_alloc(q, &mbuf[1], mbytes);
    const cudaStream_t streams[2] = {q->stream, q->aux};
    if (!rc && two &&
        (cudaEventRecord(q->ev_aux_fork, q->stream) != cudaSuccess || cudaStreamWaitEvent(q->aux, q->ev_aux_fork, 0) != cudaSuccess))
      rc = fail(SIGMO_ERR_CUDA, "stream fork failed");
    // the kernel for this batch's adjacency-row width and profile: the
    // per-lane DFS machine, or the warp-cooperative frontier join
    const bool frontier = tn.join_kernel == 1, lanes = tn.join_kernel == 2;
    const size_t smem = frontier ? sizeof(FrontWarp) * kFrontWarps
                        : lanes  ? kLaneBytesPerThread * kPhaseThreads
                                 : static_cast<size_t>(kPhaseLevels) * kPhaseThreads * (2 * 8 + 1);
    const unsigned block = frontier ? kFrontWarps * 32u : kPhaseThreads;
    void (*join_kernel)(const uint64_t*, const uint4*, uint64_t, uint64_t, const uint64_t*, const uint64_t*, const uint64_t*,
                        uint32_t, int, uint32_t, unsigned long long*, uint64_t*, unsigned long long*, JoinLimit) = nullptr;
#define SIGMO_PICK_JOIN(AWV)                                                                                \
  join_kernel = frontier ? (exact ? k_join_frontier<true, AWV> : k_join_frontier<false, AWV>)              \
                : lanes  ? (exact ? k_join_lanes<true, AWV> : k_join_lanes<false, AWV>)                    \
                         : (exact ? k_join_masks<true, AWV> : k_join_masks<false, AWV>)
    switch (data->adj_words) {
      case 1: SIGMO_PICK_JOIN(1); break;
      case 2: SIGMO_PICK_JOIN(2); break;
      default: SIGMO_PICK_JOIN(4); break;
    }
#undef SIGMO_PICK_JOIN
    if (!rc) rc = allow_max_dynamic_smem(reinterpret_cast<const void*>(join_kernel), q->device);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, q->device);
    uint64_t c = 0;
    for (uint64_t slot0 = 0; slot0 < m->total && !rc; slot0 += chunk, ++c) {
      const uint64_t cnt = std::min<uint64_t>(chunk, m->total - slot0);
      const cudaStream_t st = streams[c & 1];
      auto* masks = static_cast<uint64_t*>(mbuf[c & 1]);
      auto* recs = reinterpret_cast<uint4*>(masks + kPhaseLevels * chunk);
      unsigned long long* cursor = ctr + ((c & 1) ? 3 : 0);
      k_pair_masks<<<grid_for(cnt, 256, 148u * 16u), 256, 0, st>>>(
          planes, planes_rows, data->adj_words, pp.prog_off, prog, pp.cls, query->graph_offsets, query->qorder, query->sym,
          data->graph_offsets, data->sym, m->indices, m->pair_graph, slot0, cnt, masks, recs, skip, overflow, ctr + 2,
          m->counts);
      rc = check_launch(q, "k_pair_masks");
      if (!rc && cudaEventRecord(q->ev_masks[c & 1], st) != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "event record failed");
      if (!rc && cudaMemsetAsync(cursor, 0, 8, st) != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "memset failed");
      if (!rc) {
        // persistent CTAs; `reserve` slots stay free for a kernel running beside them
        const unsigned full = static_cast<unsigned>(sms) * tn.join_blocks_per_sm;
        const unsigned grid = full > reserve + static_cast<unsigned>(sms) ? full - reserve : full;
        // the per-lane machine and the frontier join take join_chunk slots per
        // grab; k_join_lanes takes its pool share
        join_kernel<<<grid, block, smem, st>>>(masks, recs, slot0, cnt, query->qsel, query->qsel_id, data->adj, skip,
                                               find_first, lanes ? tn.join_pool : tn.join_chunk, cursor, m->counts, tot,
                                               join_limit(q));
        rc = check_launch(q, frontier ? "k_join_frontier" : lanes ? "k_join_lanes" : "k_join_masks");
      }
    }
    // the aux stream joins the main one before its buffer is released
    if (two && (cudaEventRecord(q->ev_aux_join, q->aux) != cudaSuccess ||
                cudaStreamWaitEvent(q->stream, q->ev_aux_join, 0) != cudaSuccess))
      rc = rc ? rc : fail(SIGMO_ERR_CUDA, "stream join failed");
    dev_free(q, mbuf[0]);
    dev_free(q, mbuf[1]);
  }
  const cudaStream_t main_stream = q->stream;
  const bool side = !q->tune.overflow_serial;
  if (!rc && side) {
    // the overflow list is complete after the last Phase A of each stream: its
    // pairs run on the side stream, overlapping Phase B
    if (cudaStreamWaitEvent(q->side, q->ev_masks[0], 0) != cudaSuccess ||
        (two && cudaStreamWaitEvent(q->side, q->ev_masks[1], 0) != cudaSuccess))
      rc = fail(SIGMO_ERR_CUDA, "stream fork failed");
    q->stream = q->side;
  }
  if (!rc) {
    // the overflow list through the generic kernel
    const unsigned block = 128;
    const unsigned grid = q->tune.overflow_blocks;
    const uint32_t* list = overflow;
    const uint32_t split = q->tune.overflow_split;
    const unsigned long long* list_len = ctr + 2;
#define SIGMO_JOIN_PLANES(AWV, EX)                                                                                      \
  k_join_fast<AWV, EX, true><<<grid, block, 0, q->stream>>>(nullptr, 0, planes, planes_rows, pp.prog_off, prog, pp.cls,  \
                                                            q->opts.profile, query->graph_offsets, query->qorder,        \
                                                            query->qsel, query->qsel_id, query->sym, data->graph_offsets, \
                                                            data->adj, data->sym, m->indices, m->pair_graph, list,       \
                                                            list_len, m->total, skip, find_first, split, ctr + 1, m->counts, \
                                                            tot, join_limit(q))
    switch (data->adj_words) {
      case 1: if (exact) SIGMO_JOIN_PLANES(1, true); else SIGMO_JOIN_PLANES(1, false); break;
      case 2: if (exact) SIGMO_JOIN_PLANES(2, true); else SIGMO_JOIN_PLANES(2, false); break;
      default: if (exact) SIGMO_JOIN_PLANES(4, true); else SIGMO_JOIN_PLANES(4, false); break;
    }
#undef SIGMO_JOIN_PLANES
    rc = check_launch(q, "k_join_fast<planes>");
  }
  q->stream = main_stream;
  if (side && cudaEventRecord(q->ev_join, q->side) == cudaSuccess) cudaStreamWaitEvent(q->stream, q->ev_join, 0);
  dev_free(q, buf);
  return rc;
}

}  // namespace sigmo_b200
