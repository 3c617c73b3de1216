// device_common.cuh -- device helpers shared by the coder kernels.
//
// Included inside an anonymous namespace by every translation unit that
// instantiates the kernels (engine_kernels.cu, noalloc.cu), so each module
// carries its own copies and its own constant tables.
#pragma once

constexpr int kStageMin = 4096;
constexpr uint32_t kFlushBlock = 512;

__host__ __device__ inline int next_pow2(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}
__host__ __device__ inline int ilog2(int v) {
  int l = 0;
  while ((1 << l) < v) l++;
  return l;
}

// Overlay bucket of a key: Fibonacci hashing, logNB bits.
__device__ __forceinline__ uint32_t bucket_of(uint32_t key, int logNB) {
  return (key * 0x9E3779B1u) >> (32 - logNB);
}

__device__ inline void copy_tables(const Tables *from, Tables *dst) {
  const uint4 *src = reinterpret_cast<const uint4 *>(from);
  uint4 *d = reinterpret_cast<uint4 *>(dst);
  for (int i = threadIdx.x; i < (int)(sizeof(Tables) / 16); i += blockDim.x) d[i] = src[i];
}

// Restore a slot to its initial contents (zero, or the prelearned model).
__device__ inline void reset_slot(uint8_t *slot, const uint8_t *init_tables) {
  uint4 *d = reinterpret_cast<uint4 *>(slot);
  const size_t n = kSlotTableBytes / 16;
  if (init_tables) {
    const uint4 *src = reinterpret_cast<const uint4 *>(init_tables);
    for (size_t i = threadIdx.x; i < n; i += blockDim.x) d[i] = src[i];
  } else {
    const uint4 z = make_uint4(0, 0, 0, 0);
    for (size_t i = threadIdx.x; i < n; i += blockDim.x) d[i] = z;
  }
}

// Mixer output for one bit (Mixer::p, cucm_compress_v2.cu:636-644, then
// `if (pr < 2048) pr++`), given stretched inputs.
__device__ __forceinline__ int mix_pr(const int32_t *w, int cxt, const int smp[kOrders], const Tables *t) {
  long long sum = 0;
#pragma unroll
  for (int o = 0; o < kOrders; o++) sum += (long long)w[cxt * kOrders + o] * smp[o];
  sum >>= 16;
  int idx = sum < -2047 ? -2047 : (sum > 2048 ? 2048 : (int)sum);
  int pr = t->squash[idx + 2047];
  return pr < 2048 ? pr + 1 : pr;
}

// Coder state of a compress CTA (held by one warp; lane 0 codes).
struct Coder {
  uint32_t x1, x2;
  uint64_t head;     // bytes produced
  uint64_t flushed;  // bytes written to global
};

// Codes prm[0..n) (pr << 1 | y entries) into the shared-memory ring.  All 32
// lanes of the calling warp run the same arithmetic on the same data, so the
// control flow stays warp-uniform; lane 0 alone stores the bytes.  The ring
// never overruns: at most 4 bytes per bit are produced and at least
// stage - 4U bytes are free.  The split point x1 + floor((x2 - x1) * pr / 4096)
// is taken as the high word of (x2 - x1) * (pr << 20); it equals the
// reference's (r >> 12) * pr + ((r & 0xfff) * pr >> 12)
// (cucm_compress_v2.cu:855-856) because (r >> 12) * pr is exact.
__device__ __forceinline__ void coder_step(uint32_t e, uint32_t &x1, uint32_t &x2, uint32_t &head, uint8_t *stage,
                                           uint32_t mask, bool writer) {
  const uint32_t xm = x1 + __umulhi(x2 - x1, (e >> 1) << 20);
  if (e & 1) x2 = xm; else x1 = xm + 1;
  while ((x1 ^ x2) < 0x1000000u) {
    if (writer) stage[head & mask] = (uint8_t)(x2 >> 24);
    head++;
    x1 <<= 8;
    x2 = (x2 << 8) | 255u;
  }
}

__device__ inline void coder_run_p(Coder &c, const uint16_t *prm, uint8_t *stage, int stage_size, int n) {
  const bool writer = (threadIdx.x & 31) == 0;
  const uint32_t mask = (uint32_t)stage_size - 1;
  uint32_t x1 = c.x1, x2 = c.x2;
  uint32_t head = (uint32_t)c.head;
  const uint32_t head0 = head;
  int j = 0;
  if ((reinterpret_cast<uintptr_t>(prm) & 7) == 0) {
    for (; j + 4 <= n; j += 4) {
      const uint64_t e4 = *reinterpret_cast<const uint64_t *>(prm + j);
      coder_step((uint32_t)e4 & 0xffffu, x1, x2, head, stage, mask, writer);
      coder_step((uint32_t)(e4 >> 16) & 0xffffu, x1, x2, head, stage, mask, writer);
      coder_step((uint32_t)(e4 >> 32) & 0xffffu, x1, x2, head, stage, mask, writer);
      coder_step((uint32_t)(e4 >> 48), x1, x2, head, stage, mask, writer);
    }
  }
  for (; j < n; j++) coder_step(prm[j], x1, x2, head, stage, mask, writer);
  c.x1 = x1;
  c.x2 = x2;
  c.head += (uint32_t)(head - head0);
  __syncwarp();
}

// Warp-wide copy of complete 512-byte blocks from the ring to global.
__device__ inline void coder_flush_p(Coder &c, const uint8_t *stage, int stage_size, uint8_t *out, uint64_t cap) {
  const int lane = threadIdx.x & 31;
  const uint32_t mask = (uint32_t)stage_size - 1;
  while (c.head - c.flushed >= kFlushBlock) {
    if (c.flushed + kFlushBlock <= cap) {
      const uint32_t src = ((uint32_t)c.flushed & mask) + lane * 16;
      const uint4 v = *reinterpret_cast<const uint4 *>(stage + src);
      *reinterpret_cast<uint4 *>(out + c.flushed + lane * 16) = v;
    }
    c.flushed += kFlushBlock;
  }
  __syncwarp();
}

__device__ inline void coder_finish_p(Coder &c, uint8_t *stage, int stage_size, uint8_t *out, uint64_t cap,
                                      uint64_t *result) {
  const int lane = threadIdx.x & 31;
  const uint32_t mask = (uint32_t)stage_size - 1;
  if (lane == 0) stage[(uint32_t)c.head & mask] = (uint8_t)(c.x1 >> 24);  // flush byte, cucm_compress_v2.cu:902
  __syncwarp();
  c.head += 1;
  coder_flush_p(c, stage, stage_size, out, cap);
  for (uint64_t i = c.flushed + lane; i < c.head; i += 32)
    if (i < cap) out[i] = stage[(uint32_t)i & mask];
  if (lane == 0) *result = c.head;
  __syncwarp();
}

