/*
 * cucm_oracle.h -- CPU restatement of CuCM's chunked context-mixing coder.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker for the CUDA product in
 * cucm_b200/csrc; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.  The product never calls into it.
 *
 * Parity pinning: tests/test_oracle.py checks this restatement byte for byte
 * against the reference's own code compiled for the CPU (oracle/_ref, built
 * by oracle/make_ref.py) and against the committed golden fixtures in
 * tests/golden/, which were produced by those reference binaries.
 *
 * Every function cites the reference lines it restates
 * (cucm_compress_v2.cu / cucm_decompress_v2.cu).
 */
#ifndef CUCM_ORACLE_H
#define CUCM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CO_ORDERS 8
#define CO_SLOTS (1u << 25)
#define CO_MIXCTX 80

/* One coder model: 8 StateMaps (bit-history slots + adaptive probabilities)
 * and one Mixer (cucm_compress_v2.cu:558-679). */
typedef struct co_model {
  uint8_t *states;                      /* CO_ORDERS * CO_SLOTS bytes */
  uint32_t statep[CO_ORDERS][256];      /* 22-bit p | 10-bit count */
  int32_t w[CO_MIXCTX * CO_ORDERS];     /* 16.16 weights */
} co_model;

/* Derived tables (cucm_compress_v2.cu:681-705). */
void co_tables(int32_t squash[4096], int32_t stretch[4096], int32_t dt[1024]);
/* The 256x2 bit-history next-state table (cucm_compress_v2.cu:35-285). */
const uint8_t *co_next_state_table(void);

co_model *co_model_new(void);            /* zero model: states 0, statep 1<<31, w 0 */
void co_model_free(co_model *m);
void co_model_copy(co_model *dst, const co_model *src);

/* Host prelearn (cucm_compress_v2.cu:924-981): trains m bit-serially over
 * in[0..n) and arithmetic-codes it into out (cap bytes).  Returns the coded
 * size or (size_t)-1 if cap is too small. */
size_t co_prelearn_encode(co_model *m, const uint8_t *in, size_t n, uint8_t *out, size_t cap);
/* Raw-block replay (cucm_decompress_v2.cu:1134-1182). */
void co_prelearn_train(co_model *m, const uint8_t *in, size_t n);
/* Coded-block replay (cucm_decompress_v2.cu:1056-1132); out must be n bytes. */
void co_prelearn_decode(co_model *m, const uint8_t *in, size_t in_n, uint8_t *out, size_t n);

/* One chunk, unit-frozen GPU semantics (cucm_compress_v2.cu:711-914,
 * 1054-1107).  len = bytes of input in this chunk (<= cs; < cs only for the
 * final chunk of a stream).  Returns the payload size (coded bytes + flush
 * byte) or (size_t)-1 if cap is too small.  work must hold a copy of the
 * initial model and is left modified. */
size_t co_encode_chunk(co_model *work, const uint8_t *chunk, size_t len, size_t cs, int unit,
                       uint8_t *out, size_t cap);
/* Inverse of co_encode_chunk (cucm_decompress_v2.cu:698-1054). */
void co_decode_chunk(co_model *work, const uint8_t *payload, size_t plen, size_t len, size_t cs,
                     int unit, uint8_t *out);

/* Whole container (cucm_compress_v2.cu:1151-1250 and the CLI truncation
 * rules stay outside).  *out is malloc'd; caller frees.  threads <= 0 means
 * one per online CPU.  Returns 0 or a negative error. */
int co_compress(const uint8_t *in, size_t n, size_t cs, int unit, size_t prelearn, int batch,
                int threads, uint8_t **out, size_t *out_n);
/* The same with the fixed-model variant when `fixed` (PDF section 4.5: the
 * prelearned model codes every chunk unchanged, data bits only; header flag
 * bit 1; prelearn > 0 required).  co_compress is co_compress_ex(.., 0, ..). */
int co_compress_ex(const uint8_t *in, size_t n, size_t cs, int unit, size_t prelearn, int batch, int fixed,
                   int threads, uint8_t **out, size_t *out_n);
/* One chunk of the fixed-model variant, and its inverse; m is only read. */
size_t co_encode_chunk_fixed(const co_model *m, const uint8_t *chunk, size_t len, uint8_t *out, size_t cap);
void co_decode_chunk_fixed(const co_model *m, const uint8_t *payload, size_t plen, size_t len, uint8_t *out);
/* cucm_decompress_v2.cu:1185-1248 (and the fixed-model variant's flag). */
int co_decompress(const uint8_t *in, size_t n, int threads, uint8_t **out, size_t *out_n);

/* Upper bound on one chunk's payload for chunk size cs: every coded bit can
 * emit at most 4 bytes, plus the flush byte. */
size_t co_chunk_bound(size_t cs);

#ifdef __cplusplus
}
#endif
#endif
