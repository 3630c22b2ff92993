// Device-side helpers shared by the sigmo_b200 kernels: the reference's
// integer semantics (signature nibbles, range masks, the uint8-indexed bitset)
// under the REF_PTX and EXACT profiles.
#pragma once

#include <cstdint>

namespace sigmo_b200 {

constexpr int kProfilePtx = 0;    // SIGMO_PROFILE_REF_PTX
constexpr int kProfileX86 = 1;    // SIGMO_PROFILE_REF_X86 (stage-per-launch form only)
constexpr int kProfileExact = 2;  // SIGMO_PROFILE_EXACT
constexpr uint8_t kWildcard = 255;        // types::WILDCARD_NODE (types.hpp:23)
constexpr uint32_t kMaxQueryNodes = 64;   // join depth supported by this library
constexpr uint32_t kMaxAdjWords = 4;      // graph-local sets up to 256 vertices
constexpr uint32_t kLowOffsetLimit = 256; // REF_PTX: join bitset inert for start >= 256

// ---- Signature<PowerGraph,4>::SignatureDevice (signature.hpp:23-54) -------
__host__ __device__ __forceinline__ uint32_t sig_get(uint64_t s, uint32_t label) {
  return label < 16u ? static_cast<uint32_t>((s >> (label * 4u)) & 0xFu) : 0u;
}
// incrementLabelCount(label, 1): the counter moves only while it is < 15.
__host__ __device__ __forceinline__ uint64_t sig_inc(uint64_t s, uint32_t label) {
  if (label < 16u && sig_get(s, label) < 15u) s += 1ull << (label * 4u);
  return s;
}
// Counter l := min(count, 15) for labels < 16 (a histogram with the
// saturating increment above).
__host__ __device__ __forceinline__ uint64_t sig_put_sat(uint64_t s, uint32_t label, uint32_t count) {
  if (label < 16u) s |= static_cast<uint64_t>(count < 15u ? count : 15u) << (label * 4u);
  return s;
}

// One bit per nibble (bit 4l) set where counter l of s is non-zero.
__host__ __device__ __forceinline__ uint64_t sig_nonzero_nibbles(uint64_t s) {
  return (s | (s >> 1) | (s >> 2) | (s >> 3)) & 0x1111111111111111ull;
}

// Every counter of q <= the matching counter of d (isomorphism.hpp:103-111).
__host__ __device__ __forceinline__ bool sig_dominated(uint64_t q, uint64_t d) {
  const uint64_t E = 0x0F0F0F0F0F0F0F0Full, H = 0x1010101010101010ull;
  uint64_t even = ((d & E) | H) - (q & E);
  uint64_t odd = (((d >> 4) & E) | H) - ((q >> 4) & E);
  return ((even & odd) & H) == H;
}

// Bit-sliced "x >= c" for 32 four-bit values x (planes x0..x3, bit i of plane
// b = bit b of value i) against a scalar c in [0, 15].
__device__ __forceinline__ uint32_t ge_sliced(uint32_t x0, uint32_t x1, uint32_t x2, uint32_t x3, uint32_t c) {
  uint32_t t = (c & 1u) ? x0 : 0xFFFFFFFFu;
  t = (c & 2u) ? (x1 & t) : (x1 | t);
  t = (c & 4u) ? (x2 & t) : (x2 | t);
  t = (c & 8u) ? (x3 & t) : (x3 | t);
  return t;
}

// ---- shift semantics -------------------------------------------------------
__host__ __device__ __forceinline__ uint32_t shr32p(uint32_t v, uint32_t n) { return n >= 32u ? 0u : (v >> n); }
__host__ __device__ __forceinline__ uint32_t shl32p(uint32_t v, uint32_t n) { return n >= 32u ? 0u : (v << n); }
// x86-64 (SHL/SHR): the count is taken modulo the register width.
__host__ __device__ __forceinline__ uint32_t shr32x(uint32_t v, uint32_t n) { return v >> (n & 31u); }
__host__ __device__ __forceinline__ uint32_t shl32x(uint32_t v, uint32_t n) { return v << (n & 31u); }

// Range mask of bitset word i for the graph range [s, e)
// (CandidatesDevice::getCandidatesCount, candidates.hpp:91-99).  REF_PTX: an
// over-wide shift gives 0, so a multi-word range whose end is 32-aligned loses
// its last word.
__host__ __device__ __forceinline__ uint32_t range_mask(uint32_t i, uint32_t s, uint32_t e, int prof) {
  const uint32_t start_idx = s >> 5, end_idx = (e + 31u) >> 5;
  if (prof == kProfileExact) {
    uint32_t lo = s > (i << 5) ? s : (i << 5);
    uint32_t hi = e < ((i << 5) + 32u) ? e : ((i << 5) + 32u);
    if (lo >= hi) return 0u;
    uint32_t len = hi - lo;
    uint32_t m = len >= 32u ? 0xFFFFFFFFu : ((1u << len) - 1u);
    return m << (lo - (i << 5));
  }
  uint32_t m = 0xFFFFFFFFu;
  if (prof == kProfileX86) {  // REF_X86: an over-wide shift uses the count modulo 32
    if (start_idx == end_idx - 1u) m = shl32x(shr32x(m, 32u - (e - s)), s & 31u);
    else if (i == start_idx) m = shl32x(m, s & 31u);
    else if (i == end_idx - 1u) m = shr32x(m, 32u - (e & 31u));
    return m;
  }
  if (start_idx == end_idx - 1u) m = shl32p(shr32p(m, 32u - (e - s)), s & 31u);
  else if (i == start_idx) m = shl32p(m, s & 31u);
  else if (i == end_idx - 1u) m = shr32p(m, 32u - (e & 31u));
  return m;
}

// Bit position used by utils::detail::Bitset<uint64_t>::set/get/unset
// (utils.hpp:71-73) for vertex id x with offset `off`: the index is truncated
// to uint8_t and the subtraction is done in 32 bits; under REF_PTX a count
// >= 64 selects no bit (returns 64).
__host__ __device__ __forceinline__ uint32_t refbit_pos(uint32_t x, uint32_t off) {
  uint32_t c = (x & 0xFFu) - off;
  return c >= 64u ? 64u : c;
}
__host__ __device__ __forceinline__ uint64_t refbit(uint32_t x, uint32_t off) {
  uint32_t c = refbit_pos(x, off);
  return c >= 64u ? 0ull : (1ull << c);
}
// The same bit under the given profile: REF_X86 takes the count modulo 64, so
// the set acts on (x - off) mod 64.
__host__ __device__ __forceinline__ uint64_t refbit_prof(uint32_t x, uint32_t off, int prof) {
  if (prof == kProfileX86) return 1ull << (((x & 0xFFu) - off) & 63u);
  return refbit(x, off);
}

}  // namespace sigmo_b200
