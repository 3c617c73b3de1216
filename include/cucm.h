/*
 * cucm.h -- C ABI of the B200 CuCM coder (libcucm.so).
 *
 * The reference (OceanCT/CuCM) has no library interface: its hot path is two
 * standalone CUDA programs whose internal entry points are
 *   compress_batch()   cucm_compress_v2.cu:990-992
 *   decompressbatch()  cucm_decompress_v2.cu:898-903
 *   compress_file()    cucm_compress_v2.cu:1151-1154
 *   decompress()       cucm_decompress_v2.cu:1185
 * and whose boundary is the CLI plus the container format.  The functions
 * below are what a binding of that path would call.  Every stream produced
 * here is byte-identical to the reference's for the same input, chunk size,
 * unit length, prelearn size and batch count; every stream the reference
 * writes decodes here.
 *
 * Conventions: plain pointers and sizes, int status (0 = ok, < 0 = error,
 * see cucm_strerror), caller-owned output buffers sized with the *_bound /
 * cucm_decompressed_size queries.  A context owns one CUDA device, one
 * stream and its device memory pools; calls on one context are serialised
 * internally, distinct contexts may be used from distinct threads.  There is
 * no CPU fallback: without a usable B200 (sm_100) every compute call returns
 * CUCM_ENODEV.
 */
#ifndef CUCM_H
#define CUCM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CUCM_OK 0
#define CUCM_EINVAL (-1)     /* bad argument (size, unit, chunk size, batch) */
#define CUCM_ENOSPC (-2)     /* output buffer too small */
#define CUCM_EFORMAT (-3)    /* malformed or truncated container */
#define CUCM_ENOMEM (-4)     /* device or host allocation failed / over budget */
#define CUCM_ECUDA (-5)      /* CUDA runtime error */
#define CUCM_ENODEV (-6)     /* no usable sm_100 device */
#define CUCM_ETIMEOUT (-7)   /* a bounded device wait expired */
#define CUCM_EBUSY (-8)      /* serving queue full */
#define CUCM_ENOTFOUND (-9)  /* unknown request id */
#define CUCM_EMISMATCH (-10) /* autotuner: two execution choices gave different bytes */

/* Stream parameters: the reference's CLI flags -s -u -p -b
 * (cucm_compress_v2.cu:1288-1299).  They are stored in the container header
 * (cucm_compress_v2.cu:1197-1216) and change the bitstream. */
typedef struct cucm_params {
  uint64_t chunksize; /* -s, bytes per chunk (default 1 MiB); stored as u32 */
  uint32_t unit;      /* -u, bits per unit (default 128); multiple of 32, <= 1024 */
  uint64_t prelearn;  /* -p, bytes of host prelearn prefix (default 0) */
  uint32_t batch;     /* -b, chunks per container batch (default 100); stored as u16 */
  uint32_t format;    /* container: CUCM_FORMAT_AUTO (default), _32 or _64 */
  uint32_t fixed_model; /* 1: the fixed-model variant (see below); needs prelearn > 0; default 0 */
} cucm_params;

/* The fixed-model variant.  The paper behind the reference (its section 4.5)
 * measures CuCM with the model kept fixed after the prelearn pass -- no
 * StateMap or Mixer updates while the data is coded -- but the reference
 * ships no code for it.  Here it is a stream of its own (container flag bit
 * 1): every chunk is coded with the prelearned model, unchanged, over its
 * data bits only (no stale tail).  It is not the reference's stream; its
 * decoder is this library's.  The serving loop and the multi-GPU calls take
 * only the reference's adaptive streams. */

/* Container formats.  _32 is the reference's (cucm_compress_v2.cu:1197-1244):
 * its size fields are 32 bits, so it holds at most 4 GiB of input.  _64 has
 * no counterpart in the reference: the same chunk payloads behind a 45-byte
 * header with 64-bit sizes (first bytes ff ff ff ff 00 00 00 02, which a
 * 32-bit reader refuses) and 64-bit batch sizes and end offsets.  _AUTO
 * writes _32 up to 4 GiB of input and _64 beyond.  Decompression reads both. */
#define CUCM_FORMAT_AUTO 0u
#define CUCM_FORMAT_32 1u
#define CUCM_FORMAT_64 2u

/* Execution choices.  None of them changes a single output byte. */
typedef enum cucm_form {
  CUCM_FORM_AUTO = 0,      /* persistent unless told otherwise */
  CUCM_FORM_PLAIN = 1,     /* one kernel launch per chunk */
  CUCM_FORM_PERSISTENT = 2 /* one persistent launch, device work queue, longest first */
} cucm_form;

typedef struct cucm_tuning {
  int form;            /* cucm_form */
  int spec_bits;       /* decoder speculation depth 1..8 (0 = autotuned) */
  int max_slots;       /* cap on resident chunk slots (0 = derive from budget) */
  uint64_t hbm_budget; /* device bytes this context may hold (0 = 90% of free) */
  int kernel;          /* 0 = pipelined kernels where the unit allows, 1 = generic kernels */
  int dec_pairs;       /* decoder chunks (warp pairs) per CTA, 0 = spread over all SMs first */
  int dec_tables;      /* decoder order 0/1 tables: 0 = shared memory where it fits, 1 = slot tables */
  int cmp_ctas;        /* pipelined compressor CTAs (chunks) per SM, 1 or 2; 0 = most that fit */
  uint32_t dec_spin_limit; /* polls bounding the decoder's wait between its two warps; 0 = 2^27 (seconds).
                            * When a wait runs out the call returns CUCM_ETIMEOUT and the context stays
                            * usable; a small value makes that happen on purpose (tests). */
} cucm_tuning;

typedef struct cucm_ctx cucm_ctx;

void cucm_default_params(cucm_params *p);
const char *cucm_strerror(int status);
const char *cucm_version(void);

/* Create a context on CUDA device `device`; `tuning` may be NULL. */
int cucm_ctx_create(int device, const cucm_tuning *tuning, cucm_ctx **out);
int cucm_ctx_destroy(cucm_ctx *ctx);
int cucm_ctx_set_tuning(cucm_ctx *ctx, const cucm_tuning *tuning);
int cucm_ctx_get_tuning(cucm_ctx *ctx, cucm_tuning *tuning);

/* Largest container cucm_compress can produce for n input bytes. */
uint64_t cucm_compress_bound(uint64_t n, const cucm_params *p);
/* Original size recorded in a container header (first 4 bytes, big endian,
 * cucm_decompress_v2.cu:1298-1301; bytes 8..15 of the 64-bit container). */
int cucm_decompressed_size(const uint8_t *in, uint64_t n, uint64_t *size);

/* Whole container: the output of `cucm_compress -f IN -s -u -p -b`
 * (compress_file, cucm_compress_v2.cu:1151-1250) / of `cucm_decompress`
 * (decompress, cucm_decompress_v2.cu:1185-1248).  Host buffers. */
int cucm_compress(cucm_ctx *ctx, const uint8_t *in, uint64_t n, const cucm_params *p, uint8_t *out,
                  uint64_t cap, uint64_t *out_n);
int cucm_decompress(cucm_ctx *ctx, const uint8_t *in, uint64_t n, uint8_t *out, uint64_t cap,
                    uint64_t *out_n);

/* Same, with device-resident buffers (no host copies of the data). */
int cucm_compress_dev(cucm_ctx *ctx, const uint8_t *d_in, uint64_t n, const cucm_params *p, uint8_t *d_out,
                      uint64_t cap, uint64_t *out_n);
int cucm_decompress_dev(cucm_ctx *ctx, const uint8_t *d_in, uint64_t n, uint8_t *d_out, uint64_t cap,
                        uint64_t *out_n);

/* One batch body, no container header: `n` bytes of input split into
 * chunks of `chunksize`, coded from the zero model (compress_batch,
 * cucm_compress_v2.cu:990-1149 with sm_init = mixer_init = NULL; see
 * cucm_compress_batch_model for a prelearned model).  Output is
 * the batch body the reference writes after its u32 size field: C big-endian
 * u32 chunk end offsets followed by the chunk payloads. */
int cucm_compress_batch(cucm_ctx *ctx, const uint8_t *in, uint64_t n, uint64_t chunksize, uint32_t unit,
                        uint8_t *out, uint64_t cap, uint64_t *out_n);
/* Inverse of cucm_compress_batch (decompressbatch,
 * cucm_decompress_v2.cu:898-1054): `body` is the batch body, `out_n` the
 * number of original bytes. */
int cucm_decompress_batch(cucm_ctx *ctx, const uint8_t *body, uint64_t body_n, uint64_t chunksize, uint32_t unit,
                          uint8_t *out, uint64_t out_n);

/* An initial model: what every chunk of a stream starts from.  The
 * reference's compress_batch / decompressbatch take it as sm_init and
 * mixer_init (cucm_compress_v2.cu:990-992, cucm_decompress_v2.cu:898-903):
 * the StateMaps and Mixer trained by the host prelearn pass (prelearn,
 * cucm_compress_v2.cu:924-981), or zero.  Host memory (~450 MiB: the trained
 * tables and their device image). */
typedef struct cucm_model cucm_model;
/* The model after the prelearn pass over prefix[0..n). */
int cucm_model_prelearn(const uint8_t *prefix, uint64_t n, cucm_model **out);
/* The model a container's prelearn block defines (its prefix decoded and
 * replayed, cucm_decompress_v2.cu:1056-1182 and :1209-1219).  *out is NULL,
 * with CUCM_OK, for a container without a prelearn block. */
int cucm_model_from_container(const uint8_t *in, uint64_t n, cucm_model **out);
int cucm_model_destroy(cucm_model *m);
/* cucm_compress_batch / cucm_decompress_batch starting every chunk from `m`
 * (sm_init / mixer_init); m = NULL is the zero model.  The batch bodies of a
 * prelearned container are exactly these with the container's model. */
int cucm_compress_batch_model(cucm_ctx *ctx, const uint8_t *in, uint64_t n, uint64_t chunksize, uint32_t unit,
                              const cucm_model *m, uint8_t *out, uint64_t cap, uint64_t *out_n);
int cucm_decompress_batch_model(cucm_ctx *ctx, const uint8_t *body, uint64_t body_n, uint64_t chunksize,
                                uint32_t unit, const cucm_model *m, uint8_t *out, uint64_t out_n);

/* Multi-GPU building blocks (no counterpart in the reference, which codes on
 * one GPU).  Chunks are independent, so the chunks of one stream can be coded
 * on several GPUs and joined afterwards.
 *
 * cucm_compress_batch_dev: cucm_compress_batch_model with device buffers. */
int cucm_compress_batch_dev(cucm_ctx *ctx, const uint8_t *d_in, uint64_t n, uint64_t chunksize, uint32_t unit,
                            const cucm_model *m, uint8_t *d_out, uint64_t cap, uint64_t *out_n);
/* Join batch bodies into one container.  Body i holds counts[i] consecutive
 * chunks of the stream (what cucm_compress_batch returns for them: big-endian
 * end offsets, then payloads), the bodies in stream order; p gives chunk
 * size, unit and batch (prelearn 0), orig_size the stream's bytes.  The
 * result is byte-identical to cucm_compress of the whole stream.  Host
 * buffers and no device work; the _dev form reads device bodies and writes
 * a device container on ctx's GPU. */
int cucm_frame_bodies(const cucm_params *p, uint64_t orig_size, uint32_t nbodies, const uint8_t *const *bodies,
                      const uint64_t *body_ns, const uint32_t *counts, uint8_t *out, uint64_t cap,
                      uint64_t *out_n);
int cucm_frame_bodies_dev(cucm_ctx *ctx, const cucm_params *p, uint64_t orig_size, uint32_t nbodies,
                          const uint8_t *const *bodies, const uint64_t *body_ns, const uint32_t *counts,
                          uint8_t *d_out, uint64_t cap, uint64_t *out_n);
/* Decode chunks [first, first + count) of a container held in device memory
 * into d_out (count chunks of the chunk size, the stream's last one
 * possibly shorter); *out_n is that byte count. */
int cucm_decompress_range_dev(cucm_ctx *ctx, const uint8_t *d_in, uint64_t n, uint64_t first, uint64_t count,
                              uint8_t *d_out, uint64_t cap, uint64_t *out_n);

/* Many independent containers in one call: the batched form.  Entry i
 * reads ins[i][0..ns[i]) and writes outs[i] (caps[i] bytes), its size to
 * out_ns[i] (the size it needs when status[i] is CUCM_ENOSPC) and its status
 * to status[i]; the return value is the first failing status or CUCM_OK.
 * Each container is byte-identical to what cucm_compress makes of it alone.
 * Every chunk of every container without a prelearn prefix goes into ONE
 * persistent launch (device work queue, longest chunk first); a container
 * with a prelearn prefix has its own initial model and gets a launch of its
 * own.  Decompression batches the containers of each unit length the same
 * way.  No counterpart in the reference, which codes one file per process;
 * it replaces running compress_file / decompress once per buffer.  Host
 * buffers here, device buffers in the _dev forms. */
int cucm_compress_many(cucm_ctx *ctx, uint32_t count, const uint8_t *const *ins, const uint64_t *ns,
                       const cucm_params *p, uint8_t *const *outs, const uint64_t *caps, uint64_t *out_ns,
                       int *status);
int cucm_decompress_many(cucm_ctx *ctx, uint32_t count, const uint8_t *const *ins, const uint64_t *ns,
                         uint8_t *const *outs, const uint64_t *caps, uint64_t *out_ns, int *status);
int cucm_compress_many_dev(cucm_ctx *ctx, uint32_t count, const uint8_t *const *ins, const uint64_t *ns,
                           const cucm_params *p, uint8_t *const *outs, const uint64_t *caps, uint64_t *out_ns,
                           int *status);
int cucm_decompress_many_dev(cucm_ctx *ctx, uint32_t count, const uint8_t *const *ins, const uint64_t *ns,
                             uint8_t *const *outs, const uint64_t *caps, uint64_t *out_ns, int *status);

/* Serving loop (continuous batching).  No counterpart in the reference.
 * A server owns one device, a pool of chunk-slot tables and a buffer pool
 * carved from `hbm_budget` bytes of device memory (0 = 90% of free memory),
 * and a scheduler thread.  Requests are submitted from any thread and admitted
 * in arrival order as slots and buffer memory free up; admitted requests of
 * one kind (operation, unit length) share one persistent launch, and
 * launches on their own streams overlap on the device.  Every result is
 * byte-identical to cucm_compress / cucm_decompress of the same input.
 * Buffers passed to submit (host memory; pinned memory lets the copies run
 * asynchronously) must stay valid until poll reports the request done. */
#define CUCM_PENDING 1  /* cucm_serve_poll: the request has not finished */
typedef struct cucm_server cucm_server;
typedef enum cucm_op { CUCM_OP_COMPRESS = 0, CUCM_OP_DECOMPRESS = 1 } cucm_op;
typedef struct cucm_server_info {
  uint64_t slots;      /* chunk slots in the pool */
  uint64_t budget;     /* device bytes the server may hold */
  uint64_t completed;  /* requests finished */
  uint64_t bytes_in;   /* input bytes of finished requests */
  uint64_t bytes_out;  /* output bytes of finished requests */
  uint64_t launches;   /* engine launches so far */
  uint64_t queued;     /* requests waiting for admission */
  uint64_t inflight;   /* launches on the device */
} cucm_server_info;
int cucm_server_create(int device, uint64_t hbm_budget, const cucm_tuning *tuning, cucm_server **out);
/* Finishes every submitted request, then releases the server. */
int cucm_server_destroy(cucm_server *srv);
/* op CUCM_OP_COMPRESS: `in`/`n` is the buffer, `p` the stream parameters,
 * `out`/`cap` receives the container.  CUCM_OP_DECOMPRESS: `in`/`n` is a
 * container, `p` is ignored, `out`/`cap` receives the original bytes.
 * *id identifies the request; CUCM_EBUSY when the queue is full. */
int cucm_serve_submit(cucm_server *srv, int op, const uint8_t *in, uint64_t n, const cucm_params *p, uint8_t *out,
                      uint64_t cap, uint64_t *id);
/* Waits up to timeout_ms (0 = just look, < 0 = until done) for request `id`.
 * CUCM_OK when it is done: *status is its result (a CUCM_* code), *out_n its
 * output size (the size needed when *status is CUCM_ENOSPC), *latency_ms the
 * time from submit to completion; the id is then forgotten.  CUCM_PENDING
 * when it is still queued or running, CUCM_ENOTFOUND for an unknown id. */
int cucm_serve_poll(cucm_server *srv, uint64_t id, int timeout_ms, int *status, uint64_t *out_n, double *latency_ms);
/* Requests that may wait for admission at once (default 65536); submit
 * returns CUCM_EBUSY beyond it.  A request whose own buffers exceed the
 * server's buffer budget (a sixth of hbm_budget, at least 2 GiB) finishes
 * with status CUCM_ENOMEM instead of being admitted over the budget. */
int cucm_server_set_queue_limit(cucm_server *srv, uint32_t limit);
int cucm_server_stats(cucm_server *srv, cucm_server_info *info);

/* Device timing of the last call on this context, milliseconds (CUDA
 * events around the device work only). */
int cucm_last_device_ms(cucm_ctx *ctx, double *ms);
/* Number of kernels this context launched in the last call. */
int cucm_last_launches(cucm_ctx *ctx, uint64_t *n);

/* Measured autotuner.  No counterpart in the reference, whose launch
 * shapes are fixed.  Codes `sample` (host memory, n bytes) with `p` under
 * every candidate execution choice -- launch form; for the persistent
 * compressor, CTAs per SM (1, 2); for the persistent decoder, chunks per
 * CTA (0..5) and order 0/1 table placement; in the persistent form, warps
 * per chunk (the pipelined kernels, kernel = 0, or the generic ones,
 * kernel = 1) -- `reps`
 * times each (>= 1; the fastest repetition counts), checks that every
 * candidate gives the same container and gives the sample back (else
 * CUCM_EMISMATCH), then applies to the context and writes to *best the
 * choice with the least compress + decompress device time.  The other
 * tuning fields are kept.  results (may be null) receives up to `cap`
 * measured candidates, *count their number.  A sample with the target
 * workload's number of chunks gives choices that carry over to it. */
typedef struct cucm_tune_result {
  cucm_tuning tuning;
  double compress_ms;   /* fastest compress of the sample (< 0: a decoder candidate) */
  double decompress_ms; /* fastest decompress of the sample (< 0: a compressor candidate) */
} cucm_tune_result;
int cucm_autotune(cucm_ctx *ctx, const uint8_t *sample, uint64_t n, const cucm_params *p, int reps,
                  cucm_tune_result *results, uint32_t cap, uint32_t *count, cucm_tuning *best);

/* Figures of the last call: device_ms as above, kernel_ms the time of the
 * coder kernels alone (CUDA events around their launches), launches, and
 * the number of chunks coded. */
typedef struct cucm_stats {
  double device_ms;
  double kernel_ms;
  uint64_t launches;
  uint64_t chunks;
} cucm_stats;
int cucm_last_stats(cucm_ctx *ctx, cucm_stats *st);

/* Compress one chunk without allocating any memory.  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory when
 * they compress -- plugins whose host application owns every device
 * allocation through its own memory manager, and latency-critical paths that
 * cannot pay for cudaMalloc's implicit device synchronisation.
 * d_in: `len` input bytes in device memory (1 <= len <= chunksize); the
 * result is that chunk's payload (coded bytes and flush byte) exactly as the
 * reference codes a chunk of that length in a stream of that chunk size and
 * unit, stale tail included when len < chunksize.  d_out: device buffer of
 * `cap` bytes; *out_len receives the payload size (CUCM_ENOSPC if it is
 * larger than cap).  unit: a multiple of 32 up to 256.  stream: a
 * cudaStream_t, or NULL for the legacy default stream.  The call is
 * synchronous: it returns after the stream has finished it.
 * The only scratch is a file-scope device array holding one chunk's tables
 * (192.06 MiB per GPU, kept until the process exits), so input longer than
 * one chunk is rejected with CUCM_EINVAL.  Under lazy module loading (the
 * CUDA 12 default) a GPU reserves the array when this entry point first runs
 * on it; with CUDA_MODULE_LOADING=EAGER every context that loads the library
 * reserves it.  All calls share that array; calls that overlap on the GPU
 * race.  The first call on a device does the set-up; make it before any
 * stream capture begins. */
int cucm_compress_chunk_noalloc(const uint8_t *d_in, uint64_t len, uint64_t chunksize, uint32_t unit,
                                uint8_t *d_out, uint64_t cap, uint64_t *out_len, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* CUCM_H */
