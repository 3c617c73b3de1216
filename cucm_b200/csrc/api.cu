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
#include <new>
#include <mutex>
#include <numeric>
#include <vector>

#include "../../include/cucm.h"
#include "engine.cuh"
#include "host_model.h"
#include "model.cuh"

using namespace cucm;

namespace {

#include "container.cuh"

}  // namespace

struct cucm_model {
  cucm::ModelInit init;
  std::vector<uint8_t> image;  // slot tables in the device layout
};

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
  DevBuf d_tasks, d_results, d_queue, d_status, d_scratch, d_big, d_pack, d_body, d_out, d_tails, d_prm, d_first;
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

// A caller's model (sm_init / mixer_init), or the zero model for null.
void model_source(const cucm_model *m, ModelSource &ms) {
  if (m) {
    ms.init = m->init;
    ms.image = &m->image;
  } else {
    zero_model(ms.init);
  }
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
  cfg.dec_pairs = c->tuning.dec_pairs;
  cfg.dec_tables = c->tuning.dec_tables;
  cfg.cmp_ctas = c->tuning.cmp_ctas;
  cfg.spin_limit = c->tuning.dec_spin_limit;
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
    // work-queue counter and tail-task counter, then the tail tasks
    CK(c->d_queue.ensure(2 * sizeof(uint32_t)));
    CK(cudaMemsetAsync(c->d_queue.p, 0, 2 * sizeof(uint32_t), c->stream));
    TailTask *tails = nullptr;
    if (!decode) {
      CK(c->d_tails.ensure(sizeof(TailTask) * n));
      tails = c->d_tails.as<TailTask>();
    }
    const uint8_t *img = ms.image ? c->image.as<uint8_t>() : nullptr;
    CK(cudaEventRecord(c->evk0, c->stream));
    cudaError_t e = decode ? launch_decompress(c->d_tasks.as<ChunkTask>(), n, c->slots.as<uint8_t>(), grid, img,
                                               c->d_init.as<ModelInit>(), c->d_queue.as<uint32_t>(),
                                               c->d_status.as<uint32_t>(), cfg, c->stream, unit)
                           : launch_compress(c->d_tasks.as<ChunkTask>(), n, c->slots.as<uint8_t>(), grid, img,
                                             c->d_init.as<ModelInit>(), c->d_queue.as<uint32_t>(),
                                             c->d_status.as<uint32_t>(), cfg, c->stream, unit, tails,
                                             c->d_queue.as<uint32_t>() + 1);
    CK(e);
    CK(cudaEventRecord(c->evk1, c->stream));
    c->kernel_pending = true;
    c->launches += decode ? 1 : 2;  // the compressor's tail pass follows its engine launch
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

// A run of input bytes in device memory coded as consecutive chunks.
struct Seg {
  const uint8_t *d_in;
  uint64_t n;
};

// Chunk payloads of one engine run over several segments.
struct Encoded {
  std::vector<uint64_t> first;        // first chunk of each segment, plus the total
  std::vector<uint64_t> lens;         // payload bytes per chunk
  std::vector<const uint8_t *> src;   // payload location per chunk (device)
};

// Code every chunk of every segment in one engine run.  Payloads land in an
// optimistic scratch slot per chunk; chunks that overflow it are coded again
// with the hard bound.
int encode_chunks(cucm_ctx *c, const std::vector<Seg> &segs, uint64_t cs, uint32_t unit, const ModelSource &ms,
                  uint64_t other_bytes, Encoded &e) {
  e.first.assign(1, 0);
  for (const Seg &g : segs) e.first.push_back(e.first.back() + (g.n + cs - 1) / cs);
  const uint64_t nchunks = e.first.back();
  e.lens.assign(nchunks, 0);
  e.src.assign(nchunks, nullptr);
  if (nchunks == 0) return CUCM_OK;
  const uint64_t scap = scratch_cap(cs);
  CK(c->d_scratch.ensure(scap * nchunks));
  CK(c->d_results.ensure(sizeof(uint64_t) * nchunks));
  std::vector<ChunkTask> tasks(nchunks);
  for (size_t g = 0; g < segs.size(); g++) {
    for (uint64_t k = e.first[g]; k < e.first[g + 1]; k++) {
      const uint64_t j = k - e.first[g];
      ChunkTask &t = tasks[k];
      t.in = segs[g].d_in + j * cs;
      t.in_len = std::min<uint64_t>(cs, segs[g].n - j * cs);
      t.out = c->d_scratch.as<uint8_t>() + k * scap;
      t.out_cap = scap;
      t.cs = (uint32_t)cs;
      t.unit = unit;
      t.result = c->d_results.as<uint64_t>() + k;
    }
  }
  const std::vector<ChunkTask> orig = tasks;
  const uint64_t other = other_bytes + scap * nchunks;
  int rc = run_engine(c, false, tasks, (int)unit, ms, other);
  if (rc) return rc;
  uint32_t status = 0;
  CK(cudaMemcpyAsync(e.lens.data(), c->d_results.p, sizeof(uint64_t) * nchunks, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(&status, c->d_status.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (status & kDevBadTask) return CUCM_EINVAL;
  for (uint64_t k = 0; k < nchunks; k++) e.src[k] = orig[k].out;
  std::vector<uint64_t> redo;
  for (uint64_t k = 0; k < nchunks; k++)
    if (e.lens[k] > scap) redo.push_back(k);
  if (!redo.empty()) {
    const uint64_t hc = hard_cap(cs);
    CK(c->d_big.ensure(hc * redo.size()));
    std::vector<ChunkTask> rt;
    for (size_t i = 0; i < redo.size(); i++) {
      ChunkTask t = orig[redo[i]];
      t.out = c->d_big.as<uint8_t>() + i * hc;
      t.out_cap = hc;
      rt.push_back(t);
      e.src[redo[i]] = t.out;
    }
    rc = run_engine(c, false, rt, (int)unit, ms, other + hc * redo.size());
    if (rc) return rc;
    CK(cudaMemcpyAsync(e.lens.data(), c->d_results.p, sizeof(uint64_t) * nchunks, cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (uint64_t k : redo)
      if (e.lens[k] > hc) return CUCM_ECUDA;
  }
  return CUCM_OK;
}

// Body layout of segment g's chunks (see layout_chunks).
uint64_t layout_body(const Encoded &e, size_t g, uint32_t batch, bool with_sizes, uint8_t *base,
                     std::vector<PackEntry> *pe, bool wide = false, bool *overflow = nullptr) {
  const uint64_t f = e.first[g];
  return layout_chunks(e.lens.data() + f, e.src.data() + f, e.first[g + 1] - f, batch, with_sizes, base, pe, wide,
                       overflow);
}

// One launch packs every laid-out body.
int pack_bodies(cucm_ctx *c, const std::vector<PackEntry> &pe) {
  if (pe.empty()) return CUCM_OK;
  CK(c->d_pack.ensure(sizeof(PackEntry) * pe.size()));
  CK(cudaMemcpyAsync(c->d_pack.p, pe.data(), sizeof(PackEntry) * pe.size(), cudaMemcpyHostToDevice, c->stream));
  pack_kernel<<<(unsigned)pe.size(), 256, 0, c->stream>>>(c->d_pack.as<PackEntry>(), (uint32_t)pe.size());
  CK(cudaGetLastError());
  c->launches += 1;
  return CUCM_OK;
}

// Chunks of one container to decode: payload extents in device memory and
// where its output bytes go.
struct DecJob {
  const uint8_t *d_body;
  std::vector<uint64_t> off, len;
  uint64_t total, cs;
  uint8_t *d_out;
};

// Decode every chunk of every job in one engine run.
// The fixed-model variant (fixed_model.cuh): the model is only read, so the
// coder inputs of every chunk are computed at once (in slices of at most
// kFixedSlice input bytes: 16 bytes of inputs per input byte), then one coder
// thread per chunk codes them.  Same scratch and overflow handling as
// encode_chunks.
constexpr uint64_t kFixedSlice = 256ull << 20;

int run_fixed_encode(cucm_ctx *c, std::vector<FixedTask> &tasks, const std::vector<uint64_t> &lens) {
  // slices of consecutive tasks
  size_t k0 = 0;
  while (k0 < tasks.size()) {
    uint64_t tot = 0;
    size_t k1 = k0;
    std::vector<uint64_t> first;
    while (k1 < tasks.size() && (k1 == k0 || tot + lens[k1] <= kFixedSlice)) {
      first.push_back(tot);
      tot += lens[k1];
      k1++;
    }
    CK(c->d_prm.ensure(16 * std::max<uint64_t>(tot, 1)));
    for (size_t k = k0; k < k1; k++) tasks[k].prm = c->d_prm.as<uint16_t>() + 8 * first[k - k0];
    const uint32_t n = (uint32_t)(k1 - k0);
    CK(c->d_tasks.ensure(sizeof(FixedTask) * n));
    CK(c->d_first.ensure(sizeof(uint64_t) * n));
    CK(cudaMemcpyAsync(c->d_tasks.p, tasks.data() + k0, sizeof(FixedTask) * n, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_first.p, first.data(), sizeof(uint64_t) * n, cudaMemcpyHostToDevice, c->stream));
    CK(launch_fixed_encode(c->d_tasks.as<FixedTask>(), c->d_first.as<uint64_t>(), n, tot, c->image.as<uint8_t>(),
                           c->d_init.as<ModelInit>(), c->d_status.as<uint32_t>(), c->sm_count, c->stream));
    c->launches += 2;
    // the tasks and offsets are read by the kernels before the next slice overwrites them
    CK(cudaStreamSynchronize(c->stream));
    k0 = k1;
  }
  return CUCM_OK;
}

int encode_fixed(cucm_ctx *c, const std::vector<Seg> &segs, uint64_t cs, const ModelSource &ms, Encoded &e) {
  e.first.assign(1, 0);
  for (const Seg &g : segs) e.first.push_back(e.first.back() + (g.n + cs - 1) / cs);
  const uint64_t nchunks = e.first.back();
  e.lens.assign(nchunks, 0);
  e.src.assign(nchunks, nullptr);
  if (nchunks == 0) return CUCM_OK;
  int rc = upload_model(c, ms);
  if (rc) return rc;
  CK(c->d_status.ensure(sizeof(uint32_t)));
  CK(cudaMemsetAsync(c->d_status.p, 0, sizeof(uint32_t), c->stream));
  const uint64_t scap = scratch_cap(cs);
  CK(c->d_scratch.ensure(scap * nchunks));
  CK(c->d_results.ensure(sizeof(uint64_t) * nchunks));
  std::vector<FixedTask> tasks(nchunks);
  std::vector<uint64_t> lens(nchunks);
  for (size_t g = 0; g < segs.size(); g++) {
    for (uint64_t k = e.first[g]; k < e.first[g + 1]; k++) {
      const uint64_t j = k - e.first[g];
      FixedTask &t = tasks[k];
      t.in = segs[g].d_in + j * cs;
      t.in_len = lens[k] = std::min<uint64_t>(cs, segs[g].n - j * cs);
      t.out = c->d_scratch.as<uint8_t>() + k * scap;
      t.out_cap = scap;
      t.prm = nullptr;
      t.result = c->d_results.as<uint64_t>() + k;
      e.src[k] = t.out;
    }
  }
  collect_kernel_ms(c);
  c->chunks += nchunks;
  CK(cudaEventRecord(c->evk0, c->stream));
  rc = run_fixed_encode(c, tasks, lens);
  if (rc) return rc;
  CK(cudaMemcpyAsync(e.lens.data(), c->d_results.p, sizeof(uint64_t) * nchunks, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  std::vector<FixedTask> redo;
  std::vector<uint64_t> redo_lens, redo_k;
  for (uint64_t k = 0; k < nchunks; k++)
    if (e.lens[k] > scap) redo_k.push_back(k);
  if (!redo_k.empty()) {
    const uint64_t hc = hard_cap(cs);
    CK(c->d_big.ensure(hc * redo_k.size()));
    for (size_t i = 0; i < redo_k.size(); i++) {
      FixedTask t = tasks[redo_k[i]];
      t.out = c->d_big.as<uint8_t>() + i * hc;
      t.out_cap = hc;
      e.src[redo_k[i]] = t.out;
      redo.push_back(t);
      redo_lens.push_back(lens[redo_k[i]]);
    }
    rc = run_fixed_encode(c, redo, redo_lens);
    if (rc) return rc;
    CK(cudaMemcpyAsync(e.lens.data(), c->d_results.p, sizeof(uint64_t) * nchunks, cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (uint64_t k : redo_k)
      if (e.lens[k] > hc) return CUCM_ECUDA;
  }
  CK(cudaEventRecord(c->evk1, c->stream));
  c->kernel_pending = true;
  return CUCM_OK;
}

// Decode every chunk of fixed-model containers: one warp per chunk.
int decode_fixed(cucm_ctx *c, const std::vector<DecJob> &jobs, const ModelSource &ms) {
  std::vector<FixedTask> tasks;
  for (const DecJob &j : jobs)
    for (uint64_t k = 0; k < j.off.size(); k++) {
      FixedTask t;
      t.in = j.d_body + j.off[k];
      t.in_len = j.len[k];
      t.out = j.d_out + k * j.cs;
      t.out_cap = std::min<uint64_t>(j.cs, j.total - k * j.cs);
      t.prm = nullptr;
      t.result = nullptr;
      tasks.push_back(t);
    }
  if (tasks.empty()) return CUCM_OK;
  int rc = upload_model(c, ms);
  if (rc) return rc;
  collect_kernel_ms(c);
  c->chunks += tasks.size();
  CK(c->d_tasks.ensure(sizeof(FixedTask) * tasks.size()));
  CK(cudaMemcpyAsync(c->d_tasks.p, tasks.data(), sizeof(FixedTask) * tasks.size(), cudaMemcpyHostToDevice,
                     c->stream));
  CK(c->d_queue.ensure(2 * sizeof(uint32_t)));
  CK(cudaMemsetAsync(c->d_queue.p, 0, 2 * sizeof(uint32_t), c->stream));
  CK(cudaEventRecord(c->evk0, c->stream));
  CK(launch_fixed_decode(c->d_tasks.as<FixedTask>(), (uint32_t)tasks.size(), c->image.as<uint8_t>(),
                         c->d_init.as<ModelInit>(), c->d_queue.as<uint32_t>(), c->sm_count, c->stream));
  CK(cudaEventRecord(c->evk1, c->stream));
  c->kernel_pending = true;
  c->launches += 1;
  CK(cudaStreamSynchronize(c->stream));
  return CUCM_OK;
}

int decode_jobs(cucm_ctx *c, const std::vector<DecJob> &jobs, uint32_t unit, const ModelSource &ms,
                uint64_t other_bytes) {
  std::vector<ChunkTask> tasks;
  for (const DecJob &j : jobs) {
    for (uint64_t k = 0; k < j.off.size(); k++) {
      ChunkTask t;
      t.in = j.d_body + j.off[k];
      t.in_len = j.len[k];
      t.out = j.d_out + k * j.cs;
      t.out_cap = std::min<uint64_t>(j.cs, j.total - k * j.cs);
      t.cs = (uint32_t)j.cs;
      t.unit = unit;
      t.result = nullptr;
      tasks.push_back(t);
    }
  }
  if (tasks.empty()) return CUCM_OK;
  int rc = run_engine(c, true, tasks, (int)unit, ms, other_bytes);
  if (rc) return rc;
  uint32_t status = 0;
  CK(cudaMemcpyAsync(&status, c->d_status.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (status & kDevBadTask) return CUCM_EFORMAT;
  if (status & kDevTimeout) return CUCM_ETIMEOUT;
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
  p->format = CUCM_FORMAT_AUTO;
  p->fixed_model = 0;
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
    case CUCM_EMISMATCH: return "execution choices gave different bytes";
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

int cucm_ctx_get_tuning(cucm_ctx *c, cucm_tuning *t) {
  if (!c || !t) return CUCM_EINVAL;
  std::lock_guard<std::mutex> g(c->mu);
  *t = c->tuning;
  return CUCM_OK;
}

uint64_t cucm_compress_bound(uint64_t n, const cucm_params *p) {
  if (!p || p->chunksize == 0 || p->batch == 0) return 0;
  uint64_t body = n > p->prelearn ? n - p->prelearn : 0;
  uint64_t nchunks = (body + p->chunksize - 1) / p->chunksize;
  uint64_t nb = (nchunks + p->batch - 1) / p->batch;
  const uint64_t fw = wide_format(p, n) ? 8 : 4;
  const uint64_t hl = fw == 8 ? kHeaderBytes64 : kHeaderBytes;
  return hl + p->prelearn * 8 + 8 + fw * nb + nchunks * (fw + 32 * p->chunksize + 1);
}

int cucm_decompressed_size(const uint8_t *in, uint64_t n, uint64_t *size) {
  if (!in || !size || n < 4) return CUCM_EFORMAT;
  if (is_wide_header(in, n)) {
    if (n < 16) return CUCM_EFORMAT;
    *size = get_be64(in + 8);
    return CUCM_OK;
  }
  *size = get_be32(in);
  return CUCM_OK;
}

// Compress `count` containers that share the stream parameters `p` (the
// whole of compress_file, cucm_compress_v2.cu:1151-1250, per container).
// Containers without a prelearn prefix all start from the zero model and are
// coded in ONE engine run over all their chunks; a prelearn prefix gives a
// container its own initial model and so its own run.  `dev`: ins and outs
// are device buffers.
static int compress_containers(cucm_ctx *c, uint32_t count, const uint8_t *const *ins, const uint64_t *ns,
                               const cucm_params *p, uint8_t *const *outs, const uint64_t *caps, uint64_t *out_ns,
                               int *status, bool dev) {
  std::lock_guard<std::mutex> g(c->mu);
  CK(cudaSetDevice(c->device));
  std::vector<std::vector<uint8_t>> hdrs(count);
  std::vector<std::unique_ptr<HostModel>> models(count);
  std::vector<uint32_t> ok;
  for (uint32_t i = 0; i < count; i++) {
    out_ns[i] = 0;
    status[i] = check_params(p, ns[i]);
    if (!status[i] && ((!ins[i] && ns[i]) || !outs[i])) status[i] = CUCM_EINVAL;
    if (status[i]) continue;
    // The prelearn prefix is read on the host (it is host work in the reference).
    std::vector<uint8_t> pre;
    const uint8_t *pre_ptr = ins[i];
    if (dev && p->prelearn) {
      pre.resize(p->prelearn);
      CK(cudaMemcpy(pre.data(), ins[i], p->prelearn, cudaMemcpyDeviceToHost));
      pre_ptr = pre.data();
    }
    status[i] = make_header(pre_ptr, ns[i], p, hdrs[i], models[i]);
    if (!status[i] && caps[i] < hdrs[i].size()) {
      status[i] = CUCM_ENOSPC;
      out_ns[i] = hdrs[i].size();
    }
    if (!status[i]) ok.push_back(i);
  }
  std::vector<std::vector<uint32_t>> groups;
  if (p->prelearn == 0) {
    if (!ok.empty()) groups.push_back(ok);
  } else {
    for (uint32_t i : ok) groups.push_back({i});
  }
  timing_begin(c);
  int rc = CUCM_OK;
  for (const std::vector<uint32_t> &grp : groups) {
    ModelSource ms;
    std::vector<uint8_t> image;
    if (models[grp[0]]) {
      models[grp[0]]->to_device(image, ms.init);
      ms.image = &image;
    } else {
      zero_model(ms.init);
    }
    std::vector<Seg> segs;
    if (dev) {
      for (uint32_t i : grp) segs.push_back({ins[i] + p->prelearn, ns[i] - p->prelearn});
    } else {
      uint64_t tot = 0;
      std::vector<uint64_t> at;
      for (uint32_t i : grp) {
        at.push_back(tot);
        tot += ((ns[i] - p->prelearn) + 15) & ~15ull;
      }
      CK(c->d_body.ensure(tot ? tot : 1));
      for (size_t j = 0; j < grp.size(); j++) {
        const uint32_t i = grp[j];
        const uint64_t bn = ns[i] - p->prelearn;
        if (bn)
          CK(cudaMemcpyAsync(c->d_body.as<uint8_t>() + at[j], ins[i] + p->prelearn, bn, cudaMemcpyHostToDevice,
                             c->stream));
        segs.push_back({c->d_body.as<uint8_t>() + at[j], bn});
      }
    }
    Encoded e;
    rc = p->fixed_model ? encode_fixed(c, segs, p->chunksize, ms, e)
                        : encode_chunks(c, segs, p->chunksize, p->unit, ms, c->d_body.cap + c->d_out.cap, e);
    if (rc) break;
    std::vector<uint64_t> body(grp.size()), at(grp.size());
    uint64_t stage = 0;
    for (size_t j = 0; j < grp.size(); j++) {
      const uint32_t i = grp[j];
      bool overflow = false;
      body[j] = layout_body(e, j, p->batch, true, nullptr, nullptr, wide_format(p, ns[i]), &overflow);
      out_ns[i] = hdrs[i].size() + body[j];
      if (overflow) status[i] = CUCM_EINVAL;  // a batch past 4 GiB needs the 64-bit container
      else if (out_ns[i] > caps[i]) status[i] = CUCM_ENOSPC;
      at[j] = stage;
      stage += (body[j] + 15) & ~15ull;
    }
    if (!dev) CK(c->d_out.ensure(stage ? stage : 1));
    std::vector<PackEntry> pe;
    for (size_t j = 0; j < grp.size(); j++) {
      const uint32_t i = grp[j];
      if (status[i]) continue;
      uint8_t *base = dev ? outs[i] + hdrs[i].size() : c->d_out.as<uint8_t>() + at[j];
      layout_body(e, j, p->batch, true, base, &pe, wide_format(p, ns[i]));
    }
    rc = pack_bodies(c, pe);
    if (rc) break;
    for (size_t j = 0; j < grp.size(); j++) {
      const uint32_t i = grp[j];
      if (status[i]) continue;
      const uint64_t hl = hdrs[i].size();
      if (dev) {
        CK(cudaMemcpyAsync(outs[i], hdrs[i].data(), hl, cudaMemcpyHostToDevice, c->stream));
      } else {
        std::memcpy(outs[i], hdrs[i].data(), hl);
        if (body[j])
          CK(cudaMemcpyAsync(outs[i] + hl, c->d_out.as<uint8_t>() + at[j], body[j], cudaMemcpyDeviceToHost,
                             c->stream));
      }
    }
    CK(cudaStreamSynchronize(c->stream));
  }
  timing_end(c);
  CK(cudaStreamSynchronize(c->stream));
  if (rc) {
    for (uint32_t i : ok)
      if (!status[i]) status[i] = rc;
    return rc;
  }
  for (uint32_t i = 0; i < count; i++)
    if (status[i]) return status[i];
  return CUCM_OK;
}

int cucm_compress(cucm_ctx *c, const uint8_t *in, uint64_t n, const cucm_params *p, uint8_t *out, uint64_t cap,
                  uint64_t *out_n) {
  if (!c || !out_n || !p) return CUCM_EINVAL;
  int st = 0;
  return compress_containers(c, 1, &in, &n, p, &out, &cap, out_n, &st, false);
}

int cucm_compress_dev(cucm_ctx *c, const uint8_t *in, uint64_t n, const cucm_params *p, uint8_t *out, uint64_t cap,
                      uint64_t *out_n) {
  if (!c || !out_n || !p) return CUCM_EINVAL;
  int st = 0;
  return compress_containers(c, 1, &in, &n, p, &out, &cap, out_n, &st, true);
}

// Decompress `count` containers (decompress, cucm_decompress_v2.cu:1185-1248,
// per container).  Containers without a prelearn prefix are decoded in one
// engine run per unit length; a prelearn prefix means its own model and run.
static int decompress_containers(cucm_ctx *c, uint32_t count, const uint8_t *const *ins, const uint64_t *ns,
                                 uint8_t *const *outs, const uint64_t *caps, uint64_t *out_ns, int *status, bool dev) {
  std::lock_guard<std::mutex> g(c->mu);
  CK(cudaSetDevice(c->device));
  // The header, prelearn block and batch framing are parsed on the host.
  std::vector<std::vector<uint8_t>> host_copy(dev ? count : 0);
  std::vector<const uint8_t *> h(count);
  std::vector<Parsed> ph(count);
  std::vector<std::vector<uint64_t>> off(count), len(count);
  std::vector<uint32_t> ok;
  for (uint32_t i = 0; i < count; i++) {
    out_ns[i] = 0;
    status[i] = ins[i] ? CUCM_OK : CUCM_EINVAL;
    if (status[i]) continue;
    h[i] = ins[i];
    if (dev) {
      host_copy[i].resize(ns[i]);
      CK(cudaMemcpy(host_copy[i].data(), ins[i], ns[i], cudaMemcpyDeviceToHost));
      h[i] = host_copy[i].data();
    }
    status[i] = parse_header(h[i], ns[i], ph[i]);
    if (status[i]) continue;
    out_ns[i] = ph[i].total;
    if (ph[i].total > caps[i] || (!outs[i] && ph[i].total)) {
      status[i] = CUCM_ENOSPC;
      continue;
    }
    const uint64_t body_off = ph[i].body_off();
    const uint64_t out_body = ph[i].total - ph[i].prelearn;
    const uint64_t nchunks = (out_body + ph[i].cs - 1) / ph[i].cs;
    status[i] = parse_batches(h[i] + body_off, ns[i] - body_off, nchunks, ph[i].batch, true, off[i], len[i],
                              ph[i].wide);
    if (!status[i]) ok.push_back(i);
  }
  // groups: one per unit length for model-free containers, one per prelearned container
  std::vector<std::vector<uint32_t>> groups;
  for (uint32_t i : ok) {
    if (ph[i].prelearn) {
      groups.push_back({i});
      continue;
    }
    bool placed = false;
    for (auto &grp : groups)
      if (!ph[grp[0]].prelearn && ph[grp[0]].unit == ph[i].unit) {
        grp.push_back(i);
        placed = true;
        break;
      }
    if (!placed) groups.push_back({i});
  }
  timing_begin(c);
  int rc = CUCM_OK;
  for (const std::vector<uint32_t> &grp : groups) {
    ModelSource ms;
    std::vector<uint8_t> image, pre;
    const uint32_t i0 = grp[0];
    if (ph[i0].prelearn) {
      HostModel hm;
      pre.resize(ph[i0].prelearn);
      if (ph[i0].coded)
        hm.prelearn_decode(h[i0] + ph[i0].hdr, ph[i0].pl_len, pre.data(), ph[i0].prelearn);
      else {
        std::memcpy(pre.data(), h[i0] + ph[i0].hdr, ph[i0].prelearn);
        hm.prelearn_train(pre.data(), ph[i0].prelearn);
      }
      hm.to_device(image, ms.init);
      ms.image = &image;
    } else {
      zero_model(ms.init);
    }
    std::vector<uint64_t> bat(grp.size()), oat(grp.size());
    uint64_t btot = 0, otot = 0;
    for (size_t j = 0; j < grp.size(); j++) {
      const uint32_t i = grp[j];
      bat[j] = btot;
      oat[j] = otot;
      btot += ((ns[i] - ph[i].body_off()) + 15) & ~15ull;
      otot += ((ph[i].total - ph[i].prelearn) + 15) & ~15ull;
    }
    if (!dev) {
      CK(c->d_body.ensure(btot ? btot : 1));
      CK(c->d_out.ensure(otot ? otot : 1));
    }
    std::vector<DecJob> jobs(grp.size());
    for (size_t j = 0; j < grp.size(); j++) {
      const uint32_t i = grp[j];
      const uint64_t body_off = ph[i].body_off();
      const uint64_t body_n = ns[i] - body_off;
      DecJob &jb = jobs[j];
      if (dev) {
        jb.d_body = ins[i] + body_off;
        jb.d_out = outs[i] + ph[i].prelearn;
        if (ph[i].prelearn) CK(cudaMemcpyAsync(outs[i], pre.data(), ph[i].prelearn, cudaMemcpyHostToDevice, c->stream));
      } else {
        if (body_n)
          CK(cudaMemcpyAsync(c->d_body.as<uint8_t>() + bat[j], ins[i] + body_off, body_n, cudaMemcpyHostToDevice,
                             c->stream));
        jb.d_body = c->d_body.as<uint8_t>() + bat[j];
        jb.d_out = c->d_out.as<uint8_t>() + oat[j];
      }
      jb.off = off[i];
      jb.len = len[i];
      jb.total = ph[i].total - ph[i].prelearn;
      jb.cs = ph[i].cs;
    }
    rc = ph[i0].fixed ? decode_fixed(c, jobs, ms) : decode_jobs(c, jobs, ph[i0].unit, ms, c->d_body.cap + c->d_out.cap);
    if (rc) {
      for (uint32_t i : grp) status[i] = rc;
      if (rc == CUCM_EFORMAT) {
        rc = CUCM_OK;
        continue;
      }
      break;
    }
    if (!dev) {
      for (size_t j = 0; j < grp.size(); j++) {
        const uint32_t i = grp[j];
        if (ph[i].prelearn) std::memcpy(outs[i], pre.data(), ph[i].prelearn);
        const uint64_t ob = ph[i].total - ph[i].prelearn;
        if (ob)
          CK(cudaMemcpyAsync(outs[i] + ph[i].prelearn, jobs[j].d_out, ob, cudaMemcpyDeviceToHost, c->stream));
      }
    }
    CK(cudaStreamSynchronize(c->stream));
  }
  timing_end(c);
  CK(cudaStreamSynchronize(c->stream));
  if (rc) {
    for (uint32_t i : ok)
      if (!status[i]) status[i] = rc;
    return rc;
  }
  for (uint32_t i = 0; i < count; i++)
    if (status[i]) return status[i];
  return CUCM_OK;
}

int cucm_decompress(cucm_ctx *c, const uint8_t *in, uint64_t n, uint8_t *out, uint64_t cap, uint64_t *out_n) {
  if (!c || !in || !out_n) return CUCM_EINVAL;
  int st = 0;
  return decompress_containers(c, 1, &in, &n, &out, &cap, out_n, &st, false);
}

int cucm_decompress_dev(cucm_ctx *c, const uint8_t *in, uint64_t n, uint8_t *out, uint64_t cap, uint64_t *out_n) {
  if (!c || !in || !out_n) return CUCM_EINVAL;
  int st = 0;
  return decompress_containers(c, 1, &in, &n, &out, &cap, out_n, &st, true);
}

int cucm_model_prelearn(const uint8_t *prefix, uint64_t n, cucm_model **out) {
  if (!out || (!prefix && n)) return CUCM_EINVAL;
  *out = nullptr;
  std::unique_ptr<cucm_model> m(new (std::nothrow) cucm_model());
  if (!m) return CUCM_ENOMEM;
  try {
    HostModel hm;
    hm.prelearn_train(prefix, n);
    hm.to_device(m->image, m->init);
  } catch (const std::bad_alloc &) {
    return CUCM_ENOMEM;
  }
  *out = m.release();
  return CUCM_OK;
}

int cucm_model_from_container(const uint8_t *in, uint64_t n, cucm_model **out) {
  if (!out) return CUCM_EINVAL;
  *out = nullptr;
  Parsed ph;
  int rc = parse_header(in, n, ph);
  if (rc) return rc;
  if (!ph.prelearn) return CUCM_OK;
  std::unique_ptr<cucm_model> m(new (std::nothrow) cucm_model());
  if (!m) return CUCM_ENOMEM;
  try {
    HostModel hm;
    std::vector<uint8_t> pre(ph.prelearn);
    if (ph.coded)
      hm.prelearn_decode(in + ph.hdr, ph.pl_len, pre.data(), ph.prelearn);
    else
      hm.prelearn_train(in + ph.hdr, ph.prelearn);
    hm.to_device(m->image, m->init);
  } catch (const std::bad_alloc &) {
    return CUCM_ENOMEM;
  }
  *out = m.release();
  return CUCM_OK;
}

int cucm_model_destroy(cucm_model *m) {
  if (!m) return CUCM_EINVAL;
  delete m;
  return CUCM_OK;
}

// compress_batch of n bytes in device memory into a device body (C big-endian
// end offsets + payloads); `staged`: d_in is the context's own staging copy.
static int compress_body(cucm_ctx *c, const uint8_t *d_in, uint64_t n, uint64_t chunksize, uint32_t unit,
                         const cucm_model *m, uint8_t *d_out, uint64_t cap, uint64_t *out_n, uint8_t *h_out) {
  ModelSource ms;
  model_source(m, ms);
  Encoded e;
  int rc = encode_chunks(c, {Seg{d_in, n}}, chunksize, unit, ms, c->d_body.cap + c->d_out.cap, e);
  bool overflow = false;
  const uint64_t body_n = rc ? 0 : layout_body(e, 0, 0xffff, false, nullptr, nullptr, false, &overflow);
  *out_n = body_n;
  if (!rc && overflow) rc = CUCM_EINVAL;
  if (!rc && body_n > cap) rc = CUCM_ENOSPC;
  if (!rc && body_n) {
    uint8_t *dst = d_out;
    if (h_out) {
      CK(c->d_out.ensure(body_n));
      dst = c->d_out.as<uint8_t>();
    }
    std::vector<PackEntry> pe;
    layout_body(e, 0, 0xffff, false, dst, &pe);
    rc = pack_bodies(c, pe);
    if (!rc && h_out) CK(cudaMemcpyAsync(h_out, dst, body_n, cudaMemcpyDeviceToHost, c->stream));
  }
  return rc;
}

static int batch_args(uint64_t n, uint64_t chunksize, uint32_t unit) {
  cucm_params p;
  cucm_default_params(&p);
  p.chunksize = chunksize;
  p.unit = unit;
  p.batch = 0xffff;
  p.format = CUCM_FORMAT_32;  // a batch body's end offsets are 32-bit
  int rc = check_params(&p, n);
  if (rc) return rc;
  return (n + chunksize - 1) / chunksize > 0xffff ? CUCM_EINVAL : CUCM_OK;
}

int cucm_compress_batch_model(cucm_ctx *c, const uint8_t *in, uint64_t n, uint64_t chunksize, uint32_t unit,
                              const cucm_model *m, uint8_t *out, uint64_t cap, uint64_t *out_n) {
  if (!c || !out_n || (!in && n)) return CUCM_EINVAL;
  int rc = batch_args(n, chunksize, unit);
  if (rc) return rc;
  std::lock_guard<std::mutex> g(c->mu);
  CK(cudaSetDevice(c->device));
  timing_begin(c);
  CK(c->d_body.ensure(n ? n : 1));
  if (n) CK(cudaMemcpyAsync(c->d_body.p, in, n, cudaMemcpyHostToDevice, c->stream));
  rc = compress_body(c, c->d_body.as<uint8_t>(), n, chunksize, unit, m, nullptr, cap, out_n, out);
  timing_end(c);
  CK(cudaStreamSynchronize(c->stream));
  return rc;
}

int cucm_compress_batch_dev(cucm_ctx *c, const uint8_t *d_in, uint64_t n, uint64_t chunksize, uint32_t unit,
                            const cucm_model *m, uint8_t *d_out, uint64_t cap, uint64_t *out_n) {
  if (!c || !out_n || (!d_in && n) || !d_out) return CUCM_EINVAL;
  int rc = batch_args(n, chunksize, unit);
  if (rc) return rc;
  std::lock_guard<std::mutex> g(c->mu);
  CK(cudaSetDevice(c->device));
  timing_begin(c);
  rc = compress_body(c, d_in, n, chunksize, unit, m, d_out, cap, out_n, nullptr);
  timing_end(c);
  CK(cudaStreamSynchronize(c->stream));
  return rc;
}

int cucm_decompress_batch_model(cucm_ctx *c, const uint8_t *body, uint64_t body_n, uint64_t chunksize,
                                uint32_t unit, const cucm_model *m, uint8_t *out, uint64_t out_n) {
  if (!c || !body || (!out && out_n)) return CUCM_EINVAL;
  if (chunksize == 0 || unit < 32 || unit > (uint32_t)kMaxUnit || unit % 32) return CUCM_EINVAL;
  uint64_t nchunks = (out_n + chunksize - 1) / chunksize;
  DecJob jb;
  int rc = parse_batches(body, body_n, nchunks, (uint32_t)std::max<uint64_t>(nchunks, 1), false, jb.off, jb.len);
  if (rc) return rc;
  std::lock_guard<std::mutex> g(c->mu);
  CK(cudaSetDevice(c->device));
  ModelSource ms;
  model_source(m, ms);
  timing_begin(c);
  CK(c->d_body.ensure(body_n ? body_n : 1));
  CK(cudaMemcpyAsync(c->d_body.p, body, body_n, cudaMemcpyHostToDevice, c->stream));
  CK(c->d_out.ensure(out_n ? out_n : 1));
  jb.d_body = c->d_body.as<uint8_t>();
  jb.d_out = c->d_out.as<uint8_t>();
  jb.total = out_n;
  jb.cs = chunksize;
  rc = decode_jobs(c, {jb}, unit, ms, c->d_body.cap + c->d_out.cap);
  if (!rc && out_n) CK(cudaMemcpyAsync(out, c->d_out.p, out_n, cudaMemcpyDeviceToHost, c->stream));
  timing_end(c);
  CK(cudaStreamSynchronize(c->stream));
  return rc;
}

int cucm_compress_batch(cucm_ctx *c, const uint8_t *in, uint64_t n, uint64_t chunksize, uint32_t unit, uint8_t *out,
                        uint64_t cap, uint64_t *out_n) {
  return cucm_compress_batch_model(c, in, n, chunksize, unit, nullptr, out, cap, out_n);
}

int cucm_decompress_batch(cucm_ctx *c, const uint8_t *body, uint64_t body_n, uint64_t chunksize, uint32_t unit,
                          uint8_t *out, uint64_t out_n) {
  return cucm_decompress_batch_model(c, body, body_n, chunksize, unit, nullptr, out, out_n);
}

namespace {

// Payload extents of every chunk of `nbodies` batch bodies (C_i end offsets +
// payloads each), in stream order, from the bodies' offset tables (`tables`,
// host copies); src[k] points into the body, host or device memory alike.
int bodies_extents(uint32_t nbodies, const uint8_t *const *bodies, const uint64_t *body_ns,
                   const uint32_t *counts, const std::vector<std::vector<uint8_t>> &tables,
                   std::vector<uint64_t> &lens, std::vector<const uint8_t *> &src) {
  for (uint32_t i = 0; i < nbodies; i++) {
    const uint64_t C = counts[i];
    if (C == 0) continue;
    if (body_ns[i] < 4 * C || tables[i].size() < 4 * C) return CUCM_EFORMAT;
    uint64_t prev = 0;
    for (uint64_t k = 0; k < C; k++) {
      const uint64_t endv = get_be32(&tables[i][4 * k]);
      if (endv + 1 < 4 * C) return CUCM_EFORMAT;
      const uint64_t end = endv + 1 - 4 * C;
      if (end < prev || 4 * C + end > body_ns[i]) return CUCM_EFORMAT;
      lens.push_back(end - prev);
      src.push_back(bodies[i] + 4 * C + prev);
      prev = end;
    }
  }
  return CUCM_OK;
}

int frame_check(const cucm_params *p, uint64_t orig_size, uint32_t nbodies, const uint8_t *const *bodies,
                const uint64_t *body_ns, const uint32_t *counts, uint64_t *out_n) {
  if (!p || !out_n || (nbodies && (!bodies || !body_ns || !counts))) return CUCM_EINVAL;
  if (p->prelearn) return CUCM_EINVAL;  // a prelearn block belongs to the stream's writer
  int rc = check_params(p, orig_size);
  if (rc) return rc;
  uint64_t total = 0;
  for (uint32_t i = 0; i < nbodies; i++) {
    if (!bodies[i] && counts[i]) return CUCM_EINVAL;
    total += counts[i];
  }
  return total == (orig_size + p->chunksize - 1) / p->chunksize ? CUCM_OK : CUCM_EINVAL;
}

}  // namespace

int cucm_frame_bodies(const cucm_params *p, uint64_t orig_size, uint32_t nbodies, const uint8_t *const *bodies,
                      const uint64_t *body_ns, const uint32_t *counts, uint8_t *out, uint64_t cap,
                      uint64_t *out_n) {
  int rc = frame_check(p, orig_size, nbodies, bodies, body_ns, counts, out_n);
  if (rc) return rc;
  std::vector<std::vector<uint8_t>> tables(nbodies);
  for (uint32_t i = 0; i < nbodies; i++)
    if (counts[i]) tables[i].assign(bodies[i], bodies[i] + std::min<uint64_t>(4ull * counts[i], body_ns[i]));
  std::vector<uint64_t> lens;
  std::vector<const uint8_t *> src;
  rc = bodies_extents(nbodies, bodies, body_ns, counts, tables, lens, src);
  if (rc) return rc;
  std::vector<uint8_t> hdr;
  std::unique_ptr<HostModel> hm;
  rc = make_header(nullptr, orig_size, p, hdr, hm);
  if (rc) return rc;
  const bool wide = wide_format(p, orig_size);
  bool overflow = false;
  const uint64_t body =
      layout_chunks(lens.data(), src.data(), lens.size(), p->batch, true, nullptr, nullptr, wide, &overflow);
  if (overflow) return CUCM_EINVAL;
  *out_n = hdr.size() + body;
  if (*out_n > cap) return CUCM_ENOSPC;
  if (!out) return CUCM_EINVAL;
  std::memcpy(out, hdr.data(), hdr.size());
  std::vector<PackEntry> pe;
  layout_chunks(lens.data(), src.data(), lens.size(), p->batch, true, out + hdr.size(), &pe, wide);
  const int fw = wide ? 8 : 4;
  for (const PackEntry &e : pe) {
    if (e.len) std::memcpy(e.base + e.dst, e.src, e.len);
    for (int b = 0; b < fw; b++) e.base[e.table_at + b] = (uint8_t)(e.end_value >> (8 * (fw - 1 - b)));
    if (e.size_at != ~0ull)
      for (int b = 0; b < fw; b++) e.base[e.size_at + b] = (uint8_t)(e.batch_size >> (8 * b));
  }
  return CUCM_OK;
}

int cucm_frame_bodies_dev(cucm_ctx *c, const cucm_params *p, uint64_t orig_size, uint32_t nbodies,
                          const uint8_t *const *bodies, const uint64_t *body_ns, const uint32_t *counts,
                          uint8_t *d_out, uint64_t cap, uint64_t *out_n) {
  if (!c) return CUCM_EINVAL;
  int rc = frame_check(p, orig_size, nbodies, bodies, body_ns, counts, out_n);
  if (rc) return rc;
  std::lock_guard<std::mutex> g(c->mu);
  CK(cudaSetDevice(c->device));
  timing_begin(c);
  std::vector<std::vector<uint8_t>> tables(nbodies);
  for (uint32_t i = 0; i < nbodies; i++) {
    tables[i].resize(counts[i] ? std::min<uint64_t>(4ull * counts[i], body_ns[i]) : 0);
    if (!tables[i].empty())
      CK(cudaMemcpyAsync(tables[i].data(), bodies[i], tables[i].size(), cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  std::vector<uint64_t> lens;
  std::vector<const uint8_t *> src;
  rc = bodies_extents(nbodies, bodies, body_ns, counts, tables, lens, src);
  if (rc) return rc;
  std::vector<uint8_t> hdr;
  std::unique_ptr<HostModel> hm;
  rc = make_header(nullptr, orig_size, p, hdr, hm);
  if (rc) return rc;
  const bool wide = wide_format(p, orig_size);
  bool overflow = false;
  const uint64_t body =
      layout_chunks(lens.data(), src.data(), lens.size(), p->batch, true, nullptr, nullptr, wide, &overflow);
  if (overflow) return CUCM_EINVAL;
  *out_n = hdr.size() + body;
  if (*out_n > cap) return CUCM_ENOSPC;
  if (!d_out) return CUCM_EINVAL;
  CK(cudaMemcpyAsync(d_out, hdr.data(), hdr.size(), cudaMemcpyHostToDevice, c->stream));
  std::vector<PackEntry> pe;
  layout_chunks(lens.data(), src.data(), lens.size(), p->batch, true, d_out + hdr.size(), &pe, wide);
  rc = pack_bodies(c, pe);
  timing_end(c);
  CK(cudaStreamSynchronize(c->stream));
  return rc;
}

int cucm_decompress_range_dev(cucm_ctx *c, const uint8_t *d_in, uint64_t n, uint64_t first, uint64_t count,
                              uint8_t *d_out, uint64_t cap, uint64_t *out_n) {
  if (!c || !d_in || !out_n) return CUCM_EINVAL;
  std::lock_guard<std::mutex> g(c->mu);
  CK(cudaSetDevice(c->device));
  *out_n = 0;
  if (n < kHeaderBytes) return CUCM_EFORMAT;
  uint8_t hb[kHeaderBytes64] = {0};
  CK(cudaMemcpy(hb, d_in, std::min<uint64_t>(n, kHeaderBytes64), cudaMemcpyDeviceToHost));
  Parsed ph;
  int rc = parse_header(hb, n, ph);  // also checks that the prelearn block lies inside the n bytes
  if (rc) return rc;
  if (ph.fixed) return CUCM_EINVAL;  // the adaptive streams only
  const uint64_t body_off = ph.body_off();
  const uint64_t fw = ph.wide ? 8 : 4;
  const uint64_t out_body = ph.total - ph.prelearn;
  const uint64_t nchunks = (out_body + ph.cs - 1) / ph.cs;
  if (first > nchunks || count > nchunks - first) return CUCM_EINVAL;
  const uint64_t want = count ? std::min<uint64_t>(ph.cs * count, out_body - first * ph.cs) : 0;
  *out_n = want;
  if (want > cap) return CUCM_ENOSPC;
  if (!count) return CUCM_OK;
  if (!d_out) return CUCM_EINVAL;
  ModelSource ms;
  std::vector<uint8_t> image;
  if (ph.prelearn) {
    std::vector<uint8_t> blk(ph.pl_len), pre(ph.prelearn);
    CK(cudaMemcpy(blk.data(), d_in + ph.hdr, ph.pl_len, cudaMemcpyDeviceToHost));
    HostModel hm;
    if (ph.coded)
      hm.prelearn_decode(blk.data(), ph.pl_len, pre.data(), ph.prelearn);
    else
      hm.prelearn_train(blk.data(), ph.prelearn);
    hm.to_device(image, ms.init);
    ms.image = &image;
  } else {
    zero_model(ms.init);
  }
  // walk the batches: their size fields, and the tables of those in range
  DecJob jb;
  jb.d_body = d_in + body_off;
  jb.total = out_body - first * ph.cs;
  jb.cs = ph.cs;
  jb.d_out = d_out;
  uint64_t r = 0;
  const uint64_t body_n = n - body_off;
  for (uint64_t k0 = 0; k0 < first + count; k0 += ph.batch) {
    const uint64_t k1 = std::min<uint64_t>(k0 + ph.batch, nchunks), C = k1 - k0;
    uint8_t sz[8];
    if (r + fw > body_n) return CUCM_EFORMAT;
    CK(cudaMemcpy(sz, d_in + body_off + r, fw, cudaMemcpyDeviceToHost));
    const uint64_t bsz = get_le(sz, ph.wide);
    r += fw;
    if (bsz < fw * C || bsz > body_n - r) return CUCM_EFORMAT;
    if (k1 > first) {
      std::vector<uint8_t> tab(fw * C);
      CK(cudaMemcpy(tab.data(), d_in + body_off + r, fw * C, cudaMemcpyDeviceToHost));
      uint64_t start = 0;
      for (uint64_t k = k0; k < k1; k++) {
        const uint64_t endv = get_be(&tab[fw * (k - k0)], ph.wide);
        if (endv + 1 < fw * C) return CUCM_EFORMAT;
        const uint64_t end = endv + 1 - fw * C;
        if (end < start || end > bsz - fw * C) return CUCM_EFORMAT;
        if (k >= first && k < first + count) {
          jb.off.push_back(r + fw * C + start);
          jb.len.push_back(end - start);
        }
        start = end;
      }
    }
    r += bsz;
  }
  timing_begin(c);
  rc = decode_jobs(c, {jb}, ph.unit, ms, c->d_body.cap + c->d_out.cap);
  timing_end(c);
  CK(cudaStreamSynchronize(c->stream));
  return rc;
}

static bool many_args_ok(cucm_ctx *c, uint32_t count, const void *ins, const uint64_t *ns, const void *outs,
                         const uint64_t *caps, const uint64_t *out_ns, const int *status) {
  return c && (count == 0 || (ins && ns && outs && caps && out_ns && status));
}

int cucm_compress_many(cucm_ctx *c, uint32_t count, const uint8_t *const *ins, const uint64_t *ns,
                       const cucm_params *p, uint8_t *const *outs, const uint64_t *caps, uint64_t *out_ns,
                       int *status) {
  if (!many_args_ok(c, count, ins, ns, outs, caps, out_ns, status) || !p) return CUCM_EINVAL;
  return compress_containers(c, count, ins, ns, p, outs, caps, out_ns, status, false);
}

int cucm_compress_many_dev(cucm_ctx *c, uint32_t count, const uint8_t *const *ins, const uint64_t *ns,
                           const cucm_params *p, uint8_t *const *outs, const uint64_t *caps, uint64_t *out_ns,
                           int *status) {
  if (!many_args_ok(c, count, ins, ns, outs, caps, out_ns, status) || !p) return CUCM_EINVAL;
  return compress_containers(c, count, ins, ns, p, outs, caps, out_ns, status, true);
}

int cucm_decompress_many(cucm_ctx *c, uint32_t count, const uint8_t *const *ins, const uint64_t *ns,
                         uint8_t *const *outs, const uint64_t *caps, uint64_t *out_ns, int *status) {
  if (!many_args_ok(c, count, ins, ns, outs, caps, out_ns, status)) return CUCM_EINVAL;
  return decompress_containers(c, count, ins, ns, outs, caps, out_ns, status, false);
}

int cucm_decompress_many_dev(cucm_ctx *c, uint32_t count, const uint8_t *const *ins, const uint64_t *ns,
                             uint8_t *const *outs, const uint64_t *caps, uint64_t *out_ns, int *status) {
  if (!many_args_ok(c, count, ins, ns, outs, caps, out_ns, status)) return CUCM_EINVAL;
  return decompress_containers(c, count, ins, ns, outs, caps, out_ns, status, true);
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
