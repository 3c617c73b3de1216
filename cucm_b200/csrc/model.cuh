// model.cuh -- CuCM model constants, tables and per-bit arithmetic for sm_100a.
//
// The arithmetic restates the reference's StateMap / Mixer / coder
// (cucm_compress_v2.cu:551-705, cucm_decompress_v2.cu:519-683) exactly in
// 32-bit wrapping integer arithmetic.  Tables live in __device__ globals
// filled once per device by the host (tables.h) and are staged into shared
// memory by each CTA.
#pragma once

#include <cstdint>

// Loop-unroll hint that only the device compiler sees.
#if defined(__CUDA_ARCH__)
#define CUCM_UNROLL _Pragma("unroll")
#else
#define CUCM_UNROLL
#endif

namespace cucm {

constexpr int kOrders = 8;
constexpr uint32_t kSlotBits = 25;
constexpr uint32_t kSlots = 1u << kSlotBits;   // per hashed order
constexpr int kMixCtx = 80;
constexpr int kMaxUnit = 1024;                 // largest supported unit length (bits)
constexpr uint32_t kFnvBasis = 2166136261u;
constexpr uint32_t kFnvPrime = 16777619u;

// Table placement inside one chunk slot (bytes).  Orders 0 and 1 are
// collision-free under the 25-bit hash, so they are stored exactly by their
// context instead of by slot: order 0 by h0 (1..255), order 1 by
// (previous byte << 8 | h0).  Orders 2..7 keep the full 2^25-slot layout.
constexpr uint64_t kOrder0Bytes = 256;
constexpr uint64_t kOrder1Bytes = 65536;
constexpr uint64_t kOrder1Off = kOrder0Bytes;
constexpr uint64_t kHashedOff = kOrder0Bytes + kOrder1Bytes;
constexpr uint64_t kSlotTableBytes = kHashedOff + 6ull * kSlots;

__host__ __device__ inline uint64_t table_offset(int order) {
  return order == 0 ? 0 : (order == 1 ? kOrder1Off : kHashedOff + (uint64_t)(order - 2) * kSlots);
}

// Squash/stretch/dt tables and the next-state table, in a layout that can be
// copied into shared memory with 16-byte vector moves.
struct Tables {
  int16_t stretch[4096];
  uint16_t squash[4096];
  uint16_t dt[1024];
  uint8_t nex[256][2];
};

// StateMap::update restated (cucm_compress_v2.cu:592-601): the int
// conversions of the reference become explicit 32-bit wraparound.
__host__ __device__ inline uint32_t statep_next(uint32_t v, int y, uint32_t dtv) {
  uint32_t cnt = v & 1023u;
  int32_t err = (int32_t)(((uint32_t)y << 22) - (v >> 10));
  uint32_t adj = ((uint32_t)(err >> 3) * dtv) & 0xfffffc00u;
  return v + adj + (cnt < 1023u ? 1u : 0u);
}

// Binary arithmetic coder split point (cucm_compress_v2.cu:855-856).
__host__ __device__ inline uint32_t coder_mid(uint32_t x1, uint32_t x2, uint32_t pr) {
  uint32_t r = x2 - x1;
  return x1 + (r >> 12) * pr + (((r & 0xfffu) * pr) >> 12);
}

// The reference's table key of order `o` for a bit: order 0 keyed by h0,
// order 1 by (c1 << 8 | h0), orders >= 2 by the 25-bit FNV-1 slot.
struct BitKeys {
  uint32_t k[kOrders];
};

// Context keys of one bit (cucm_compress_v2.cu:723-747).  h0 is the partial
// byte with a leading 1, hist[i-1] the i-th previous byte (0 before the
// chunk start).  FNV over h[0..o], low 25 bits; 32-bit arithmetic is exact
// because only low bits are kept.
__host__ __device__ inline void bit_keys(uint32_t h0, const uint32_t hist[7], BitKeys &out) {
  uint32_t acc = (kFnvBasis ^ h0) * kFnvPrime;
  out.k[0] = h0;
  out.k[1] = (hist[0] << 8) | h0;
  acc = (acc ^ hist[0]) * kFnvPrime;
CUCM_UNROLL
  for (int o = 2; o < kOrders; o++) {
    acc = (acc ^ hist[o - 1]) * kFnvPrime;
    out.k[o] = acc & (kSlots - 1);
  }
}

// Same keys from a 64-bit history word: byte i of `h` (i = 0 is the least
// significant) is the (i+1)-th previous byte.
__host__ __device__ inline void bit_keys64(uint32_t h0, uint64_t h, BitKeys &out) {
  uint32_t hist[7];
CUCM_UNROLL
  for (int i = 0; i < 7; i++) hist[i] = (uint32_t)(h >> (8 * i)) & 0xffu;
  bit_keys(h0, hist, out);
}

}  // namespace cucm
