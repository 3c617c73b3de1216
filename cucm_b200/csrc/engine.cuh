// engine.cuh -- device-side job descriptors and host-side engine interface.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "model.cuh"

namespace cucm {

// Per-chunk model initial state (statep + mixer weights); the slot tables
// hold the bit-history states.
struct ModelInit {
  uint32_t statep[kOrders][256];
  int32_t w[kMixCtx * kOrders];
};

// One chunk of work.  All pointers are device pointers.
struct ChunkTask {
  const uint8_t *in;     // compress: chunk input; decompress: chunk payload
  uint8_t *out;          // compress: payload scratch; decompress: output bytes
  uint64_t in_len;       // compress: input bytes; decompress: payload bytes
  uint64_t out_cap;      // compress: scratch capacity; decompress: output bytes (len)
  uint32_t cs;           // chunk size of the stream (format field)
  uint32_t unit;         // unit length in bits (format field)
  uint64_t *result;      // compress: payload length written here (or > cap on overflow)
};

// The stale tail of a chunk handed from a persistent compress CTA to the tail
// pass: the coder state after the chunk's last data unit, and the unit buffer
// the reference keeps re-coding up to the chunk end
// (cucm_compress_v2.cu:850-852).
struct TailTask {
  uint8_t *out;       // payload; bytes [0, head) are written
  uint64_t cap;       // payload capacity
  uint64_t *result;   // payload length goes here
  uint64_t head;      // bytes produced so far
  uint64_t bits;      // stale bits still to code: prm[j % unit] for j < bits
  uint32_t x1, x2;
  uint32_t unit;
  uint32_t pad;
  uint16_t prm[256];  // the last data unit's buffer (units up to 256 bits)
};

// One chunk of a fixed-model launch (the variant without online updates).
// compress: in = the chunk's bytes, prm = room for its coder inputs (8 u16
// per byte, 16-byte aligned), out = payload scratch; decompress: in = the
// payload, out = the chunk's bytes.
struct FixedTask {
  const uint8_t *in;
  uint64_t in_len;   // compress: chunk bytes; decompress: payload bytes
  uint8_t *out;
  uint64_t out_cap;  // compress: payload capacity; decompress: chunk bytes
  uint16_t *prm;
  uint64_t *result;  // compress: payload length
};

// Status words written by the kernels (per launch).
enum DevStatus : uint32_t {
  kDevOk = 0,
  kDevOverflow = 1,      // some chunk's payload exceeded its scratch capacity
  kDevBadTask = 2,       // malformed task (unit/size out of range)
  kDevTimeout = 4,       // a bounded wait between the warps of a chunk gave up
};

struct EngineConfig {
  int threads = 256;           // CTA size (multiple of 64)
  int spec_bits = 4;           // decoder speculation depth (1..8); never changes output
  bool generic = false;        // force the generic (non-pipelined) kernels
  int sm_count = 0;            // SMs of the device (0 = query)
  int dec_pairs = 0;           // decoder chunks per CTA (0 = spread over all SMs first)
  int dec_tables = 0;          // decoder order 0/1 tables: 0 = shared memory where it fits, 1 = slot tables
  int cmp_ctas = 0;            // pipelined compressor CTAs per SM (0 = derived)
  uint32_t spin_limit = 0;     // decoder: polls bounding the wait for a published round (0 = default)
};

cudaError_t upload_tables();  // once per device (current device)

// Launch helpers (all asynchronous on `stream`).
// slots: nslots chunk-slot tables of kSlotTableBytes each, already holding
// the initial model states.  init_tables: a clean copy to restore slots from
// between chunks (nullptr = restore to zero).  queue: one u32 counter.
// tails: room for ntasks tail tasks and a zeroed u32 counter (tail_count),
// or null to code every stale tail in place (the plain form passes null).
cudaError_t launch_compress(const ChunkTask *d_tasks, uint32_t ntasks, uint8_t *slots, uint32_t nslots,
                            const uint8_t *init_tables, const ModelInit *d_init, uint32_t *d_queue,
                            uint32_t *d_status, const EngineConfig &cfg, cudaStream_t stream, int unit,
                            TailTask *tails = nullptr, uint32_t *tail_count = nullptr);
cudaError_t launch_decompress(const ChunkTask *d_tasks, uint32_t ntasks, uint8_t *slots, uint32_t nslots,
                              const uint8_t *init_tables, const ModelInit *d_init, uint32_t *d_queue,
                              uint32_t *d_status, const EngineConfig &cfg, cudaStream_t stream, int unit);

// Fixed-model variant: coder inputs of every byte of every task (first[]:
// prefix sums of the chunk lengths, total bytes), then one coder thread per
// task; and the decoder, one warp per task from a zeroed queue counter.
// image / d_init: the prelearned model in the device layout.
cudaError_t launch_fixed_encode(const FixedTask *d_tasks, const uint64_t *d_first, uint32_t ntasks, uint64_t total,
                                const uint8_t *image, const ModelInit *d_init, uint32_t *d_status, int sm_count,
                                cudaStream_t stream);
cudaError_t launch_fixed_decode(const FixedTask *d_tasks, uint32_t ntasks, const uint8_t *image,
                                const ModelInit *d_init, uint32_t *d_queue, int sm_count, cudaStream_t stream);

size_t compress_smem_bytes(int unit);
// Chunk slots of the engine that run at once on one SM.
int engine_slots_per_sm(bool decode, int unit, const EngineConfig &cfg);
int compress_threads(int unit);
size_t decompress_smem_bytes(int unit, int spec_bits);

}  // namespace cucm
