// api.cu -- libcucm: the C ABI (include/cucm.h) over the device engine.
//
// Host responsibilities, kept in C++ like the reference's host code:
//   * container writer/reader (compress_file cucm_compress_v2.cu:1151-1250,
//     decompress cucm_decompress_v2.cu:1185-1248): 21-byte big-endian header,
//     prelearn block, per batch a host-order (little-endian) u32 size, C
//     big-endian u32 chunk end offsets and the chunk payloads;
//   * the optional bit-serial prelearn pass (host_model.h);
//   * device pools (chunk-slot tables, scratch, tasks), the work order
//     (longest first) and the launch form (plain or persistent);
//   * the pack step that lays the chunk payloads out as batches.
// The chunk payloads never depend on the batch size (-b) -- only the framing
// does -- so every chunk of a container goes to the device in one launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>
#include <vector>

#include "../../include/cucm.h"
#include "engine.cuh"
#include "host_model.h"
#include "model.cuh"

using namespace cucm;

namespace {

constexpr uint64_t kHeaderBytes = 21;

// ---------------------------------------------------------------------------
// Pack kernel: one CTA per chunk copies its payload from scratch into the
// container, writes its big-endian end offset, and the first chunk of a batch
// writes the batch's little-endian size field.
struct PackEntry {
  uint64_t src;        // scratch offset of the payload
  uint64_t dst;        // container offset of the payload
  uint64_t len;        // payload bytes
  uint64_t table_at;   // container offset of this chunk's end-offset field
  uint32_t end_value;  // big-endian field value
  uint32_t batch_size; // valid when size_at != ~0
  uint64_t size_at;    // container offset of the batch size field or ~0
};

__global__ void pack_kernel(const PackEntry *e, uint32_t n, const uint8_t *scratch, uint8_t *dst) {
  const uint32_t k = blockIdx.x;
  if (k >= n) return;
  const PackEntry p = e[k];
  const uint8_t *s = scratch + p.src;
  uint8_t *d = dst + p.dst;
  for (uint64_t i = threadIdx.x; i < p.len; i += blockDim.x) d[i] = s[i];
  if (threadIdx.x == 0) {
    uint8_t *t = dst + p.table_at;
    t[0] = (uint8_t)(p.end_value >> 24);
    t[1] = (uint8_t)(p.end_value >> 16);
    t[2] = (uint8_t)(p.end_value >> 8);
    t[3] = (uint8_t)p.end_value;
    if (p.size_at != ~0ull) {
      uint8_t *z = dst + p.size_at;
      z[0] = (uint8_t)p.batch_size;
      z[1] = (uint8_t)(p.batch_size >> 8);
      z[2] = (uint8_t)(p.batch_size >> 16);
      z[3] = (uint8_t)(p.batch_size >> 24);
    }
  }
}

struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
  cudaError_t ensure(size_t n) {
    if (n <= cap) return cudaSuccess;
    release();
    size_t want = n < 256 ? 256 : n;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
      p = nullptr;
      return e;
    }
    cap = want;
    return cudaSuccess;
  }
  template <typename T>
  T *as() const {
    return reinterpret_cast<T *>(p);
  }
};

inline void put_be32(uint8_t *p, uint32_t v) {
  p[0] = (uint8_t)(v >> 24);
  p[1] = (uint8_t)(v >> 16);
  p[2] = (uint8_t)(v >> 8);
  p[3] = (uint8_t)v;
}
inline uint32_t get_be32(const uint8_t *p) {
  return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
}
inline uint32_t get_le32(const uint8_t *p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

uint64_t scratch_cap(uint64_t cs) {
  // Typical payloads stay below ~1.1x the chunk; 2x + 4 KiB leaves margin.
  // A chunk that still overflows is re-coded with the hard bound.
  uint64_t c = 2 * cs + 4096;
  uint64_t hard = 32 * cs + 16;
  return ((c < hard ? c : hard) + 15) & ~15ull;
}
uint64_t hard_cap(uint64_t cs) { return (32 * cs + 1 + 15) & ~15ull; }

}  // namespace

struct cucm_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<cudaStream_t> side;  // plain form
  cucm_tuning tuning{};
  std::mutex mu;
  int sm_count = 0;
  DevBuf slots;
  uint32_t nslots = 0;
  DevBuf image;    // prelearned slot image (when used)
  DevBuf d_init;   // ModelInit
  DevBuf d_tasks, d_results, d_queue, d_status, d_scratch, d_pack, d_body, d_out;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t evk0 = nullptr, evk1 = nullptr;  // around the engine launches
  double last_ms = 0.0;
  double kernel_ms = 0.0;
  bool kernel_pending = false;
  uint64_t launches = 0;
  uint64_t chunks = 0;
  bool timing_open = false;
};

namespace {

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return CUCM_OK;
  if (e == cudaErrorMemoryAllocation) return CUCM_ENOMEM;
  if (e == cudaErrorNoDevice || e == cudaErrorInvalidDevice || e == cudaErrorNoKernelImageForDevice ||
      e == cudaErrorInsufficientDriver)
    return CUCM_ENODEV;
  return CUCM_ECUDA;
}

#define CK(call)                        \
  do {                                  \
    cudaError_t e_ = (call);            \
    if (e_ != cudaSuccess) return cuda_status(e_); \
  } while (0)

struct ModelSource {
  ModelInit init;
  const std::vector<uint8_t> *image = nullptr;  // nullptr: zero tables
};

void zero_model(ModelInit &mi) {
  for (int o = 0; o < kOrders; o++)
    for (int s = 0; s < 256; s++) mi.statep[o][s] = 1u << 31;
  std::memset(mi.w, 0, sizeof mi.w);
}

uint64_t budget_bytes(cucm_ctx *c) {
  size_t freeb = 0, total = 0;
  cudaMemGetInfo(&freeb, &total);
  uint64_t b = c->tuning.hbm_budget ? c->tuning.hbm_budget : (uint64_t)(0.9 * (double)freeb);
  return b;
}

// Make sure the context holds at least `want` slot tables.
int ensure_slots(cucm_ctx *c, uint32_t want, uint64_t other_bytes) {
  if (want <= c->nslots) return CUCM_OK;
  c->slots.release();
  c->nslots = 0;
  uint64_t b = budget_bytes(c);
  uint64_t room = b > other_bytes ? b - other_bytes : 0;
  uint64_t fit = room / kSlotTableBytes;
  if (fit == 0) return CUCM_ENOMEM;
  uint32_t n = (uint32_t)std::min<uint64_t>(want, fit);
  CK(c->slots.ensure((size_t)n * kSlotTableBytes));
  c->nslots = n;
  return CUCM_OK;
}

// Chunks the engine runs at once on the whole device.
int resident_chunks(cucm_ctx *c, bool decode, int unit, const EngineConfig &cfg) {
  return engine_slots_per_sm(decode, unit, cfg) * c->sm_count;
}

int fill_slots(cucm_ctx *c, uint32_t n, const ModelSource &ms) {
  if (!ms.image) {
    CK(cudaMemsetAsync(c->slots.p, 0, (size_t)n * kSlotTableBytes, c->stream));
  } else {
    for (uint32_t i = 0; i < n; i++)
      CK(cudaMemcpyAsync(c->slots.as<uint8_t>() + (size_t)i * kSlotTableBytes, c->image.p, kSlotTableBytes,
                         cudaMemcpyDeviceToDevice, c->stream));
  }
  return CUCM_OK;
}

int upload_model(cucm_ctx *c, const ModelSource &ms) {
  CK(c->d_init.ensure(sizeof(ModelInit)));
  CK(cudaMemcpyAsync(c->d_init.p, &ms.init, sizeof(ModelInit), cudaMemcpyHostToDevice, c->stream));
  if (ms.image) {
    CK(c->image.ensure(kSlotTableBytes));
    CK(cudaMemcpyAsync(c->image.p, ms.image->data(), kSlotTableBytes, cudaMemcpyHostToDevice, c->stream));
  }
  return CUCM_OK;
}

void timing_begin(cucm_ctx *c) {
  c->launches = 0;
  c->chunks = 0;
  c->kernel_ms = 0.0;
  c->kernel_pending = false;
  cudaEventRecord(c->ev0, c->stream);
  c->timing_open = true;
}
// Adds the engine time recorded by the last run_engine (the stream must have
// been synchronised past evk1).
void collect_kernel_ms(cucm_ctx *c) {
  if (!c->kernel_pending) return;
  float ms = 0;
  if (cudaEventElapsedTime(&ms, c->evk0, c->evk1) == cudaSuccess) c->kernel_ms += ms;
  c->kernel_pending = false;
}

void timing_end(cucm_ctx *c) {
  if (!c->timing_open) return;
  cudaEventRecord(c->ev1, c->stream);
  cudaEventSynchronize(c->ev1);
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  c->last_ms = ms;
  collect_kernel_ms(c);
  c->timing_open = false;
}

// Run the engine over `tasks` (host copies; pointers are device pointers).
// Results (payload lengths for compress) are written into tasks[i].result
// targets on the device; the caller reads them back.
int run_engine(cucm_ctx *c, bool decode, std::vector<ChunkTask> &tasks, int unit, const ModelSource &ms,
               uint64_t other_bytes) {
  const uint32_t n = (uint32_t)tasks.size();
  if (n == 0) return CUCM_OK;
  EngineConfig cfg;
  cfg.spec_bits = c->tuning.spec_bits > 0 ? c->tuning.spec_bits : 4;
  cfg.generic = c->tuning.kernel == 1;
  cfg.sm_count = c->sm_count;
  const int form = c->tuning.form == CUCM_FORM_PLAIN ? CUCM_FORM_PLAIN : CUCM_FORM_PERSISTENT;

  int rc = upload_model(c, ms);
  if (rc) return rc;
  CK(c->d_status.ensure(sizeof(uint32_t)));
  CK(cudaMemsetAsync(c->d_status.p, 0, sizeof(uint32_t), c->stream));
  collect_kernel_ms(c);
  c->chunks += n;

  if (form == CUCM_FORM_PERSISTENT) {
    // Longest first: model work grows with the input bytes, coder work with
    // the chunk size (stale tail included).
    std::stable_sort(tasks.begin(), tasks.end(), [&](const ChunkTask &a, const ChunkTask &b) {
      uint64_t la = (decode ? a.out_cap : a.in_len) * 4 + a.cs;
      uint64_t lb = (decode ? b.out_cap : b.in_len) * 4 + b.cs;
      return la > lb;
    });
    uint32_t want = std::min<uint32_t>(n, (uint32_t)resident_chunks(c, decode, unit, cfg));
    if (c->tuning.max_slots > 0) want = std::min<uint32_t>(want, (uint32_t)c->tuning.max_slots);
    rc = ensure_slots(c, want, other_bytes);
    if (rc) return rc;
    uint32_t grid = std::min<uint32_t>(want, c->nslots);
    rc = fill_slots(c, grid, ms);
    if (rc) return rc;
    CK(c->d_tasks.ensure(sizeof(ChunkTask) * n));
    CK(cudaMemcpyAsync(c->d_tasks.p, tasks.data(), sizeof(ChunkTask) * n, cudaMemcpyHostToDevice, c->stream));
    CK(c->d_queue.ensure(sizeof(uint32_t)));
    CK(cudaMemsetAsync(c->d_queue.p, 0, sizeof(uint32_t), c->stream));
    const uint8_t *img = ms.image ? c->image.as<uint8_t>() : nullptr;
    CK(cudaEventRecord(c->evk0, c->stream));
    cudaError_t e = decode ? launch_decompress(c->d_tasks.as<ChunkTask>(), n, c->slots.as<uint8_t>(), grid, img,
                                               c->d_init.as<ModelInit>(), c->d_queue.as<uint32_t>(),
                                               c->d_status.as<uint32_t>(), cfg, c->stream, unit)
                           : launch_compress(c->d_tasks.as<ChunkTask>(), n, c->slots.as<uint8_t>(), grid, img,
                                             c->d_init.as<ModelInit>(), c->d_queue.as<uint32_t>(),
                                             c->d_status.as<uint32_t>(), cfg, c->stream, unit);
    CK(e);
    CK(cudaEventRecord(c->evk1, c->stream));
    c->kernel_pending = true;
    c->launches += 1;
  } else {
    // Plain form: one single-CTA launch per chunk.  At most 128 grids can be
    // resident on the device, so chunks are spread over <= 128 streams, each
    // with its own slot, cleared before every launch.
    uint32_t want = std::min<uint32_t>(n, 128u);
    if (c->tuning.max_slots > 0) want = std::min<uint32_t>(want, (uint32_t)c->tuning.max_slots);
    rc = ensure_slots(c, want, other_bytes);
    if (rc) return rc;
    uint32_t S = std::min<uint32_t>(want, c->nslots);
    while (c->side.size() < S) {
      cudaStream_t st;
      CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
      c->side.push_back(st);
    }
    CK(c->d_tasks.ensure(sizeof(ChunkTask) * n));
    CK(cudaMemcpyAsync(c->d_tasks.p, tasks.data(), sizeof(ChunkTask) * n, cudaMemcpyHostToDevice, c->stream));
    CK(c->d_queue.ensure(sizeof(uint32_t) * n));
    CK(cudaMemsetAsync(c->d_queue.p, 0, sizeof(uint32_t) * n, c->stream));
    cudaEvent_t fork;
    CK(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    CK(cudaEventRecord(c->evk0, c->stream));
    CK(cudaEventRecord(fork, c->stream));
    for (uint32_t s = 0; s < S; s++) CK(cudaStreamWaitEvent(c->side[s], fork, 0));
    const uint8_t *img = ms.image ? c->image.as<uint8_t>() : nullptr;
    for (uint32_t i = 0; i < n; i++) {
      uint32_t s = i % S;
      uint8_t *slot = c->slots.as<uint8_t>() + (size_t)s * kSlotTableBytes;
      if (img)
        CK(cudaMemcpyAsync(slot, img, kSlotTableBytes, cudaMemcpyDeviceToDevice, c->side[s]));
      else
        CK(cudaMemsetAsync(slot, 0, kSlotTableBytes, c->side[s]));
      cudaError_t e = decode ? launch_decompress(c->d_tasks.as<ChunkTask>() + i, 1, slot, 1, img,
                                                 c->d_init.as<ModelInit>(), c->d_queue.as<uint32_t>() + i,
                                                 c->d_status.as<uint32_t>(), cfg, c->side[s], unit)
                             : launch_compress(c->d_tasks.as<ChunkTask>() + i, 1, slot, 1, img,
                                               c->d_init.as<ModelInit>(), c->d_queue.as<uint32_t>() + i,
                                               c->d_status.as<uint32_t>(), cfg, c->side[s], unit);
      CK(e);
      c->launches += 1;
    }
    for (uint32_t s = 0; s < S; s++) {
      cudaEvent_t done;
      CK(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
      CK(cudaEventRecord(done, c->side[s]));
      CK(cudaStreamWaitEvent(c->stream, done, 0));
      cudaEventDestroy(done);
    }
    cudaEventDestroy(fork);
    CK(cudaEventRecord(c->evk1, c->stream));
    c->kernel_pending = true;
  }
  return CUCM_OK;
}

// Validate stream parameters the way the reference's container can hold them.
int check_params(const cucm_params *p, uint64_t n) {
  if (!p) return CUCM_EINVAL;
  if (p->chunksize == 0 || p->chunksize > 0xffffffffull) return CUCM_EINVAL;
  if (p->unit < 32 || p->unit > (uint32_t)kMaxUnit || p->unit % 32) return CUCM_EINVAL;
  if (p->batch == 0 || p->batch > 0xffff) return CUCM_EINVAL;
  if (p->prelearn > n) return CUCM_EINVAL;
  if (n > 0xffffffffull) return CUCM_EINVAL;  // header field is 32 bits
  return CUCM_OK;
}

struct Layout2 {
  uint64_t nchunks, nbatches, total;
  std::vector<uint64_t> lens;
};

// Encode every chunk of `d_body[0..n)` and pack the batches at d_dst.
// Returns the container body size (everything after the prelearn block).
int encode_and_pack(cucm_ctx *c, const uint8_t *d_body, uint64_t n, uint64_t cs, uint32_t unit, uint32_t batch,
                    const ModelSource &ms, bool with_sizes, uint8_t *d_dst, uint64_t dst_cap, uint64_t *body_n,
                    std::vector<uint64_t> *lens_out) {
  const uint64_t nchunks = (n + cs - 1) / cs;
  *body_n = 0;
  if (nchunks == 0) return CUCM_OK;
  std::vector<uint64_t> scap(nchunks), soff(nchunks);
  uint64_t tot = 0;
  for (uint64_t k = 0; k < nchunks; k++) {
    scap[k] = scratch_cap(cs);
    soff[k] = tot;
    tot += scap[k];
  }
  CK(c->d_scratch.ensure(tot));
  CK(c->d_results.ensure(sizeof(uint64_t) * nchunks));
  std::vector<ChunkTask> tasks(nchunks);
  for (uint64_t k = 0; k < nchunks; k++) {
    ChunkTask &t = tasks[k];
    t.in = d_body + k * cs;
    t.in_len = std::min<uint64_t>(cs, n - k * cs);
    t.out = c->d_scratch.as<uint8_t>() + soff[k];
    t.out_cap = scap[k];
    t.cs = (uint32_t)cs;
    t.unit = unit;
    t.result = c->d_results.as<uint64_t>() + k;
  }
  uint64_t other = tot + c->d_body.cap + c->d_out.cap;
  int rc = run_engine(c, false, tasks, (int)unit, ms, other);
  if (rc) return rc;
  std::vector<uint64_t> lens(nchunks);
  uint32_t status = 0;
  CK(cudaMemcpyAsync(lens.data(), c->d_results.p, sizeof(uint64_t) * nchunks, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(&status, c->d_status.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (status & kDevBadTask) return CUCM_EINVAL;
  // Re-code chunks whose payload overflowed the optimistic scratch.
  std::vector<uint64_t> redo;
  for (uint64_t k = 0; k < nchunks; k++)
    if (lens[k] > scap[k]) redo.push_back(k);
  DevBuf big;
  std::vector<uint64_t> big_off(nchunks, ~0ull);
  if (!redo.empty()) {
    uint64_t btot = 0;
    for (uint64_t k : redo) {
      big_off[k] = btot;
      btot += hard_cap(cs);
    }
    CK(big.ensure(btot));
    std::vector<ChunkTask> rt;
    for (uint64_t k : redo) {
      ChunkTask t = tasks[0];
      t.in = d_body + k * cs;
      t.in_len = std::min<uint64_t>(cs, n - k * cs);
      t.out = big.as<uint8_t>() + big_off[k];
      t.out_cap = hard_cap(cs);
      t.cs = (uint32_t)cs;
      t.unit = unit;
      t.result = c->d_results.as<uint64_t>() + k;
      rt.push_back(t);
    }
    rc = run_engine(c, false, rt, (int)unit, ms, other + btot);
    if (rc) return rc;
    CK(cudaMemcpyAsync(lens.data(), c->d_results.p, sizeof(uint64_t) * nchunks, cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (uint64_t k : redo)
      if (lens[k] > hard_cap(cs)) return CUCM_ECUDA;
  }
  // Layout of the batches (cudaencodefinal, cucm_compress_v2.cu:880-914).
  const uint64_t nb = (nchunks + batch - 1) / batch;
  std::vector<PackEntry> pe(nchunks);
  uint64_t w = 0;
  for (uint64_t b = 0; b < nb; b++) {
    uint64_t k0 = b * batch, k1 = std::min<uint64_t>(k0 + batch, nchunks), C = k1 - k0;
    uint64_t bsz = 4 * C;
    for (uint64_t k = k0; k < k1; k++) bsz += lens[k];
    uint64_t size_at = w;
    if (with_sizes) w += 4;
    uint64_t table = w;
    w += 4 * C;
    uint64_t acc = 4 * C - 1;
    for (uint64_t k = k0; k < k1; k++) {
      acc += lens[k];
      PackEntry &p = pe[k];
      bool in_big = big_off[k] != ~0ull;
      p.src = in_big ? big_off[k] : soff[k];
      p.dst = w;
      p.len = lens[k];
      p.table_at = table + 4 * (k - k0);
      p.end_value = (uint32_t)acc;
      p.size_at = (k == k0 && with_sizes) ? size_at : ~0ull;
      p.batch_size = (uint32_t)bsz;
      w += lens[k];
    }
  }
  if (w > dst_cap) return CUCM_ENOSPC;
  CK(c->d_pack.ensure(sizeof(PackEntry) * nchunks));
  CK(cudaMemcpyAsync(c->d_pack.p, pe.data(), sizeof(PackEntry) * nchunks, cudaMemcpyHostToDevice, c->stream));
  if (redo.empty()) {
    pack_kernel<<<(unsigned)nchunks, 256, 0, c->stream>>>(c->d_pack.as<PackEntry>(), (uint32_t)nchunks,
                                                           c->d_scratch.as<uint8_t>(), d_dst);
    c->launches += 1;
  } else {
    // two sources: pack the overflowed chunks from the big scratch separately
    std::vector<PackEntry> a, bb;
    for (uint64_t k = 0; k < nchunks; k++) (big_off[k] != ~0ull ? bb : a).push_back(pe[k]);
    DevBuf pa, pb;
    CK(pa.ensure(sizeof(PackEntry) * std::max<size_t>(a.size(), 1)));
    CK(pb.ensure(sizeof(PackEntry) * std::max<size_t>(bb.size(), 1)));
    CK(cudaMemcpyAsync(pa.p, a.data(), sizeof(PackEntry) * a.size(), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(pb.p, bb.data(), sizeof(PackEntry) * bb.size(), cudaMemcpyHostToDevice, c->stream));
    if (!a.empty())
      pack_kernel<<<(unsigned)a.size(), 256, 0, c->stream>>>(pa.as<PackEntry>(), (uint32_t)a.size(),
                                                             c->d_scratch.as<uint8_t>(), d_dst);
    pack_kernel<<<(unsigned)bb.size(), 256, 0, c->stream>>>(pb.as<PackEntry>(), (uint32_t)bb.size(),
                                                            big.as<uint8_t>(), d_dst);
    c->launches += 2;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
  }
  CK(cudaGetLastError());
  *body_n = w;
  if (lens_out) *lens_out = lens;
  return CUCM_OK;
}

// Container header + prelearn block.  Also produces the initial model.
int make_header(const uint8_t *in, uint64_t n, const cucm_params *p, std::vector<uint8_t> &hdr,
                std::unique_ptr<HostModel> &hm) {
  std::vector<uint8_t> pl;
  uint64_t coded = 0;
  if (p->prelearn > 0) {
    hm.reset(new HostModel());
    coded = hm->prelearn_encode(in, p->prelearn, pl);
  }
  const bool raw = p->prelearn <= coded;  // cucm_compress_v2.cu:1217-1223
  const uint64_t pl_len = raw ? p->prelearn : coded;
  hdr.assign(kHeaderBytes + pl_len, 0);
  put_be32(&hdr[0], (uint32_t)n);
  hdr[4] = (uint8_t)(p->batch >> 8);
  hdr[5] = (uint8_t)p->batch;
  hdr[6] = (uint8_t)(p->unit >> 8);
  hdr[7] = (uint8_t)p->unit;
  put_be32(&hdr[8], (uint32_t)p->chunksize);
  put_be32(&hdr[12], (uint32_t)coded);
  put_be32(&hdr[16], (uint32_t)p->prelearn);
  hdr[20] = raw ? 0 : 1;
  if (pl_len) std::memcpy(&hdr[kHeaderBytes], raw ? in : pl.data(), pl_len);
  return CUCM_OK;
}

struct Parsed {
  uint64_t total, cs, prelearn, pl_coded, pl_len;
  uint32_t batch, unit;
  int coded;
};

int parse_header(const uint8_t *in, uint64_t n, Parsed &h) {
  if (!in || n < kHeaderBytes) return CUCM_EFORMAT;
  h.total = get_be32(in);
  h.batch = ((uint32_t)in[4] << 8) | in[5];
  h.unit = ((uint32_t)in[6] << 8) | in[7];
  h.cs = get_be32(in + 8);
  h.pl_coded = get_be32(in + 12);
  h.prelearn = get_be32(in + 16);
  h.coded = in[20];
  if (h.cs == 0 || h.batch == 0 || h.unit < 32 || h.unit > (uint32_t)kMaxUnit || h.unit % 32) return CUCM_EFORMAT;
  if (h.prelearn > h.total) return CUCM_EFORMAT;
  h.pl_len = h.coded ? h.pl_coded : h.prelearn;
  if (kHeaderBytes + h.pl_len > n) return CUCM_EFORMAT;
  return CUCM_OK;
}

// Chunk payload extents of the batches that follow the prelearn block
// (cucm_decompress_v2.cu:1223-1237).  Offsets are relative to `body`.
int parse_batches(const uint8_t *body, uint64_t body_n, uint64_t nchunks, uint32_t batch, bool with_sizes,
                  std::vector<uint64_t> &off, std::vector<uint64_t> &len) {
  off.resize(nchunks);
  len.resize(nchunks);
  uint64_t r = 0;
  const uint64_t nb = (nchunks + batch - 1) / batch;
  for (uint64_t b = 0; b < nb; b++) {
    uint64_t k0 = b * batch, k1 = std::min<uint64_t>(k0 + batch, nchunks), C = k1 - k0;
    uint64_t bsz;
    if (with_sizes) {
      if (r + 4 > body_n) return CUCM_EFORMAT;
      bsz = get_le32(body + r);
      r += 4;
    } else {
      bsz = body_n - r;
    }
    if (bsz < 4 * C || r + bsz > body_n) return CUCM_EFORMAT;
    const uint64_t pay0 = r + 4 * C;
    const uint64_t pay_n = bsz - 4 * C;
    uint64_t start = 0;
    for (uint64_t k = k0; k < k1; k++) {
      uint64_t endv = get_be32(body + r + 4 * (k - k0));
      if (endv + 1 < 4 * C) return CUCM_EFORMAT;
      uint64_t end = endv + 1 - 4 * C;
      if (end < start || end > pay_n) return CUCM_EFORMAT;
      off[k] = pay0 + start;
      len[k] = end - start;
      start = end;
    }
    r += bsz;
  }
  return CUCM_OK;
}

int decode_chunks(cucm_ctx *c, const uint8_t *d_body, const std::vector<uint64_t> &off,
                  const std::vector<uint64_t> &len, uint64_t total, uint64_t cs, uint32_t unit, const ModelSource &ms,
                  uint8_t *d_out) {
  const uint64_t nchunks = off.size();
  if (nchunks == 0) return CUCM_OK;
  std::vector<ChunkTask> tasks(nchunks);
  for (uint64_t k = 0; k < nchunks; k++) {
    ChunkTask &t = tasks[k];
    t.in = d_body + off[k];
    t.in_len = len[k];
    t.out = d_out + k * cs;
    t.out_cap = std::min<uint64_t>(cs, total - k * cs);
    t.cs = (uint32_t)cs;
    t.unit = unit;
    t.result = nullptr;
  }
  int rc = run_engine(c, true, tasks, (int)unit, ms, c->d_body.cap + c->d_out.cap);
  if (rc) return rc;
  uint32_t status = 0;
  CK(cudaMemcpyAsync(&status, c->d_status.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (status & kDevBadTask) return CUCM_EFORMAT;
  return CUCM_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI

extern "C" {

void cucm_default_params(cucm_params *p) {
  if (!p) return;
  p->chunksize = 1024 * 1024;  // cucm_compress_v2.cu:1308
  p->unit = 128;               // cucm_compress_v2.cu:1306
  p->prelearn = 0;
  p->batch = 100;              // cucm_compress_v2.cu:1312
}

const char *cucm_strerror(int s) {
  switch (s) {
    case CUCM_OK: return "ok";
    case CUCM_EINVAL: return "invalid argument";
    case CUCM_ENOSPC: return "output buffer too small";
    case CUCM_EFORMAT: return "malformed or truncated container";
    case CUCM_ENOMEM: return "out of memory or over the HBM budget";
    case CUCM_ECUDA: return "CUDA runtime error";
    case CUCM_ENODEV: return "no usable sm_100 CUDA device";
    case CUCM_ETIMEOUT: return "bounded device wait expired";
    case CUCM_EBUSY: return "serving queue full";
    case CUCM_ENOTFOUND: return "unknown request";
    default: return "unknown error";
  }
}

const char *cucm_version(void) { return "cucm-b200 0.1"; }

int cucm_ctx_create(int device, const cucm_tuning *tuning, cucm_ctx **out) {
  if (!out) return CUCM_EINVAL;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return CUCM_ENODEV;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return CUCM_ENODEV;
  if (prop.major != 10) return CUCM_ENODEV;  // built for sm_100a only
  CK(cudaSetDevice(device));
  std::unique_ptr<cucm_ctx> c(new cucm_ctx());
  c->device = device;
  c->sm_count = prop.multiProcessorCount;
  if (tuning) c->tuning = *tuning;
  CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  CK(cudaEventCreate(&c->ev0));
  CK(cudaEventCreate(&c->ev1));
  CK(cudaEventCreate(&c->evk0));
  CK(cudaEventCreate(&c->evk1));
  CK(upload_tables());
  CK(cudaDeviceSynchronize());
  *out = c.release();
  return CUCM_OK;
}

int cucm_ctx_destroy(cucm_ctx *c) {
  if (!c) return CUCM_EINVAL;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  for (cudaStream_t s : c->side) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
  cudaStreamDestroy(c->stream);
  cudaEventDestroy(c->ev0);
  cudaEventDestroy(c->ev1);
  cudaEventDestroy(c->evk0);
  cudaEventDestroy(c->evk1);
  delete c;
  return CUCM_OK;
}

int cucm_ctx_set_tuning(cucm_ctx *c, const cucm_tuning *t) {
  if (!c || !t) return CUCM_EINVAL;
  std::lock_guard<std::mutex> g(c->mu);
  c->tuning = *t;
  return CUCM_OK;
}

uint64_t cucm_compress_bound(uint64_t n, const cucm_params *p) {
  if (!p || p->chunksize == 0 || p->batch == 0) return 0;
  uint64_t body = n > p->prelearn ? n - p->prelearn : 0;
  uint64_t nchunks = (body + p->chunksize - 1) / p->chunksize;
  uint64_t nb = (nchunks + p->batch - 1) / p->batch;
  return kHeaderBytes + p->prelearn * 8 + 8 + 4 * nb + nchunks * (4 + 32 * p->chunksize + 1);
}

int cucm_decompressed_size(const uint8_t *in, uint64_t n, uint64_t *size) {
  if (!in || !size || n < 4) return CUCM_EFORMAT;
  *size = get_be32(in);
  return CUCM_OK;
}

static int compress_impl(cucm_ctx *c, const uint8_t *in, uint64_t n, const cucm_params *p, uint8_t *out,
                         uint64_t cap, uint64_t *out_n, bool dev) {
  if (!c || !out_n || (!in && n) || !out) return CUCM_EINVAL;
  int rc = check_params(p, n);
  if (rc) return rc;
  std::lock_guard<std::mutex> g(c->mu);
  CK(cudaSetDevice(c->device));
  // The prelearn prefix is read on the host (it is host work in the reference).
  std::vector<uint8_t> pre;
  const uint8_t *pre_ptr = in;
  if (dev && p->prelearn) {
    pre.resize(p->prelearn);
    CK(cudaMemcpy(pre.data(), in, p->prelearn, cudaMemcpyDeviceToHost));
    pre_ptr = pre.data();
  }
  std::vector<uint8_t> hdr;
  std::unique_ptr<HostModel> hm;
  rc = make_header(pre_ptr, n, p, hdr, hm);
  if (rc) return rc;
  ModelSource ms;
  std::vector<uint8_t> image;
  if (hm) {
    hm->to_device(image, ms.init);
    ms.image = &image;
  } else {
    zero_model(ms.init);
  }
  const uint64_t body_in = n - p->prelearn;
  const uint64_t hl = hdr.size();
  if (cap < hl) return CUCM_ENOSPC;
  timing_begin(c);
  const uint8_t *d_body;
  uint8_t *d_dst;
  uint64_t dst_cap;
  if (dev) {
    d_body = in + p->prelearn;
    d_dst = out + hl;
    dst_cap = cap - hl;
  } else {
    CK(c->d_body.ensure(body_in ? body_in : 1));
    if (body_in)
      CK(cudaMemcpyAsync(c->d_body.p, in + p->prelearn, body_in, cudaMemcpyHostToDevice, c->stream));
    d_body = c->d_body.as<uint8_t>();
    uint64_t nchunks = (body_in + p->chunksize - 1) / p->chunksize;
    uint64_t est = body_in * 2 + nchunks * (8 + 4096) + 64;
    CK(c->d_out.ensure(est));
    d_dst = c->d_out.as<uint8_t>();
    dst_cap = c->d_out.cap;
  }
  uint64_t body_n = 0;
  rc = encode_and_pack(c, d_body, body_in, p->chunksize, p->unit, p->batch, ms, true, d_dst, dst_cap, &body_n,
                       nullptr);
  if (rc == CUCM_ENOSPC && !dev) {
    // grow the device staging buffer to the hard bound and retry
    CK(c->d_out.ensure(cucm_compress_bound(n, p)));
    rc = encode_and_pack(c, d_body, body_in, p->chunksize, p->unit, p->batch, ms, true, c->d_out.as<uint8_t>(),
                         c->d_out.cap, &body_n, nullptr);
  }
  if (rc) {
    timing_end(c);
    return rc;
  }
  if (hl + body_n > cap) {
    timing_end(c);
    return CUCM_ENOSPC;
  }
  if (dev) {
    CK(cudaMemcpyAsync(out, hdr.data(), hl, cudaMemcpyHostToDevice, c->stream));
  } else {
    std::memcpy(out, hdr.data(), hl);
    if (body_n) CK(cudaMemcpyAsync(out + hl, c->d_out.p, body_n, cudaMemcpyDeviceToHost, c->stream));
  }
  timing_end(c);
  CK(cudaStreamSynchronize(c->stream));
  *out_n = hl + body_n;
  return CUCM_OK;
}

int cucm_compress(cucm_ctx *c, const uint8_t *in, uint64_t n, const cucm_params *p, uint8_t *out, uint64_t cap,
                  uint64_t *out_n) {
  return compress_impl(c, in, n, p, out, cap, out_n, false);
}

int cucm_compress_dev(cucm_ctx *c, const uint8_t *in, uint64_t n, const cucm_params *p, uint8_t *out, uint64_t cap,
                      uint64_t *out_n) {
  return compress_impl(c, in, n, p, out, cap, out_n, true);
}

static int decompress_impl(cucm_ctx *c, const uint8_t *in, uint64_t n, uint8_t *out, uint64_t cap,
                           uint64_t *out_n, bool dev) {
  if (!c || !in || !out_n) return CUCM_EINVAL;
  std::lock_guard<std::mutex> g(c->mu);
  CK(cudaSetDevice(c->device));
  // The header, prelearn block and batch framing are parsed on the host.
  std::vector<uint8_t> host_copy;
  const uint8_t *h = in;
  if (dev) {
    host_copy.resize(n);
    CK(cudaMemcpy(host_copy.data(), in, n, cudaMemcpyDeviceToHost));
    h = host_copy.data();
  }
  Parsed ph;
  int rc = parse_header(h, n, ph);
  if (rc) return rc;
  if (ph.total > cap || (!out && ph.total)) return CUCM_ENOSPC;
  ModelSource ms;
  std::vector<uint8_t> image;
  std::vector<uint8_t> pre(ph.prelearn);
  if (ph.prelearn) {
    HostModel hm;
    if (ph.coded)
      hm.prelearn_decode(h + kHeaderBytes, ph.pl_len, pre.data(), ph.prelearn);
    else {
      std::memcpy(pre.data(), h + kHeaderBytes, ph.prelearn);
      hm.prelearn_train(pre.data(), ph.prelearn);
    }
    hm.to_device(image, ms.init);
    ms.image = &image;
  } else {
    zero_model(ms.init);
  }
  const uint64_t body_off = kHeaderBytes + ph.pl_len;
  const uint64_t body_n = n - body_off;
  const uint64_t out_body = ph.total - ph.prelearn;
  const uint64_t nchunks = (out_body + ph.cs - 1) / ph.cs;
  std::vector<uint64_t> off, len;
  rc = parse_batches(h + body_off, body_n, nchunks, ph.batch, true, off, len);
  if (rc) return rc;
  timing_begin(c);
  const uint8_t *d_body;
  uint8_t *d_o;
  if (dev) {
    d_body = in + body_off;
    d_o = out + ph.prelearn;
    if (ph.prelearn) CK(cudaMemcpyAsync(out, pre.data(), ph.prelearn, cudaMemcpyHostToDevice, c->stream));
  } else {
    CK(c->d_body.ensure(body_n ? body_n : 1));
    if (body_n) CK(cudaMemcpyAsync(c->d_body.p, in + body_off, body_n, cudaMemcpyHostToDevice, c->stream));
    d_body = c->d_body.as<uint8_t>();
    CK(c->d_out.ensure(out_body ? out_body : 1));
    d_o = c->d_out.as<uint8_t>();
  }
  rc = decode_chunks(c, d_body, off, len, out_body, ph.cs, ph.unit, ms, d_o);
  if (rc) {
    timing_end(c);
    return rc;
  }
  if (!dev) {
    if (ph.prelearn) std::memcpy(out, pre.data(), ph.prelearn);
    if (out_body) CK(cudaMemcpyAsync(out + ph.prelearn, d_o, out_body, cudaMemcpyDeviceToHost, c->stream));
  }
  timing_end(c);
  CK(cudaStreamSynchronize(c->stream));
  *out_n = ph.total;
  return CUCM_OK;
}

int cucm_decompress(cucm_ctx *c, const uint8_t *in, uint64_t n, uint8_t *out, uint64_t cap, uint64_t *out_n) {
  return decompress_impl(c, in, n, out, cap, out_n, false);
}

int cucm_decompress_dev(cucm_ctx *c, const uint8_t *in, uint64_t n, uint8_t *out, uint64_t cap, uint64_t *out_n) {
  return decompress_impl(c, in, n, out, cap, out_n, true);
}

int cucm_compress_batch(cucm_ctx *c, const uint8_t *in, uint64_t n, uint64_t chunksize, uint32_t unit, uint8_t *out,
                        uint64_t cap, uint64_t *out_n) {
  if (!c || !out_n || (!in && n)) return CUCM_EINVAL;
  cucm_params p;
  cucm_default_params(&p);
  p.chunksize = chunksize;
  p.unit = unit;
  p.batch = 0xffff;
  int rc = check_params(&p, n);
  if (rc) return rc;
  uint64_t nchunks = (n + chunksize - 1) / chunksize;
  if (nchunks > 0xffff) return CUCM_EINVAL;
  std::lock_guard<std::mutex> g(c->mu);
  CK(cudaSetDevice(c->device));
  ModelSource ms;
  zero_model(ms.init);
  timing_begin(c);
  CK(c->d_body.ensure(n ? n : 1));
  if (n) CK(cudaMemcpyAsync(c->d_body.p, in, n, cudaMemcpyHostToDevice, c->stream));
  CK(c->d_out.ensure(n * 2 + nchunks * (8 + 4096) + 64));
  uint64_t body_n = 0;
  rc = encode_and_pack(c, c->d_body.as<uint8_t>(), n, chunksize, unit, 0xffff, ms, false, c->d_out.as<uint8_t>(),
                       c->d_out.cap, &body_n, nullptr);
  if (rc) {
    timing_end(c);
    return rc;
  }
  if (body_n > cap) {
    timing_end(c);
    return CUCM_ENOSPC;
  }
  if (body_n) CK(cudaMemcpyAsync(out, c->d_out.p, body_n, cudaMemcpyDeviceToHost, c->stream));
  timing_end(c);
  CK(cudaStreamSynchronize(c->stream));
  *out_n = body_n;
  return CUCM_OK;
}

int cucm_decompress_batch(cucm_ctx *c, const uint8_t *body, uint64_t body_n, uint64_t chunksize, uint32_t unit,
                          uint8_t *out, uint64_t out_n) {
  if (!c || !body || (!out && out_n)) return CUCM_EINVAL;
  if (chunksize == 0 || unit < 32 || unit > (uint32_t)kMaxUnit || unit % 32) return CUCM_EINVAL;
  uint64_t nchunks = (out_n + chunksize - 1) / chunksize;
  std::vector<uint64_t> off, len;
  int rc = parse_batches(body, body_n, nchunks, (uint32_t)std::max<uint64_t>(nchunks, 1), false, off, len);
  if (rc) return rc;
  std::lock_guard<std::mutex> g(c->mu);
  CK(cudaSetDevice(c->device));
  ModelSource ms;
  zero_model(ms.init);
  timing_begin(c);
  CK(c->d_body.ensure(body_n ? body_n : 1));
  CK(cudaMemcpyAsync(c->d_body.p, body, body_n, cudaMemcpyHostToDevice, c->stream));
  CK(c->d_out.ensure(out_n ? out_n : 1));
  rc = decode_chunks(c, c->d_body.as<uint8_t>(), off, len, out_n, chunksize, unit, ms, c->d_out.as<uint8_t>());
  if (rc) {
    timing_end(c);
    return rc;
  }
  if (out_n) CK(cudaMemcpyAsync(out, c->d_out.p, out_n, cudaMemcpyDeviceToHost, c->stream));
  timing_end(c);
  CK(cudaStreamSynchronize(c->stream));
  return CUCM_OK;
}

int cucm_compress_many(cucm_ctx *c, uint32_t count, const uint8_t *const *ins, const uint64_t *ns,
                       const cucm_params *p, uint8_t *const *outs, const uint64_t *caps, uint64_t *out_ns,
                       int *status) {
  if (!c || (count && (!ins || !ns || !outs || !caps || !out_ns || !status))) return CUCM_EINVAL;
  int first = CUCM_OK;
  for (uint32_t i = 0; i < count; i++) {
    status[i] = cucm_compress(c, ins[i], ns[i], p, outs[i], caps[i], &out_ns[i]);
    if (status[i] && !first) first = status[i];
  }
  return first;
}

int cucm_decompress_many(cucm_ctx *c, uint32_t count, const uint8_t *const *ins, const uint64_t *ns,
                         uint8_t *const *outs, const uint64_t *caps, uint64_t *out_ns, int *status) {
  if (!c || (count && (!ins || !ns || !outs || !caps || !out_ns || !status))) return CUCM_EINVAL;
  int first = CUCM_OK;
  for (uint32_t i = 0; i < count; i++) {
    status[i] = cucm_decompress(c, ins[i], ns[i], outs[i], caps[i], &out_ns[i]);
    if (status[i] && !first) first = status[i];
  }
  return first;
}

int cucm_last_device_ms(cucm_ctx *c, double *ms) {
  if (!c || !ms) return CUCM_EINVAL;
  *ms = c->last_ms;
  return CUCM_OK;
}

int cucm_last_launches(cucm_ctx *c, uint64_t *n) {
  if (!c || !n) return CUCM_EINVAL;
  *n = c->launches;
  return CUCM_OK;
}

int cucm_last_stats(cucm_ctx *c, cucm_stats *st) {
  if (!c || !st) return CUCM_EINVAL;
  st->device_ms = c->last_ms;
  st->kernel_ms = c->kernel_ms;
  st->launches = c->launches;
  st->chunks = c->chunks;
  return CUCM_OK;
}

}  // extern "C"
