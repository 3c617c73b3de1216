// serve.cu -- the serving loop: continuous batching of compress and
// decompress requests on one GPU (cucm_server_*, cucm_serve_*).
//
// The reference has no server; it codes one file per process.  Here a
// request is one buffer to compress into a container, or one container to
// decompress, submitted from any host thread.  A scheduler thread owns the
// device:
//
//   * admission: queued requests are admitted in arrival order while chunk
//     slots (the 192 MiB bit-history tables, a fixed pool carved from the HBM
//     budget) and buffer memory (a CUDA memory pool, also under the budget)
//     are free.  Requests that arrive while others run are admitted as soon
//     as slots free up -- there is no waiting for the GPU to drain;
//   * a launch takes all admissible requests of one kind (operation, unit
//     length, no prelearn model) and runs every chunk of them in one
//     persistent engine launch on its own stream, over a contiguous run of
//     slots; launches on different streams overlap on the device;
//   * compress launches finish in a second step: the payload lengths come
//     back, the container layout is computed on the host, one pack kernel
//     writes every container and the bytes go back to the caller;
//   * slots are cleared on the launch's stream before they return to the
//     pool, so a slot is always clean when a launch takes it.
//
// Every output is byte-identical to the single-call API's: a chunk's bytes
// depend only on its own input and the stream parameters.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/cucm.h"
#include "engine.cuh"
#include "host_model.h"
#include "model.cuh"

using namespace cucm;

namespace {

#include "container.cuh"

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct Req {
  uint64_t id = 0;
  int op = 0;
  const uint8_t *in = nullptr;
  uint64_t n = 0;
  cucm_params p{};
  uint8_t *out = nullptr;
  uint64_t cap = 0;
  bool done = false;
  int status = 0;
  uint64_t out_n = 0;
  double t_submit = 0, t_admit = 0, t_done = 0;
  // prepared on the scheduler thread
  bool prepared = false;
  uint32_t unit = 0;
  uint64_t cs = 0;
  uint64_t nchunks = 0;
  std::vector<uint8_t> hdr;             // compress: header + prelearn block
  std::unique_ptr<HostModel> hm;        // compress: prelearned model
  Parsed ph{};                          // decompress
  std::vector<uint64_t> off, len;       // decompress: payload extents in the body
  std::vector<uint8_t> pre;             // decompress: prelearn bytes
  uint64_t body_off = 0, body_n = 0;    // input body (after header + prelearn block)
  uint64_t out_body = 0;                // decompress: output bytes after the prelearn prefix
};

enum Phase { kRun = 0, kRedo = 1, kFinish = 2 };

struct Launch {
  int op = 0;
  uint32_t unit = 0;
  bool model = false;  // prelearned model (single request)
  std::vector<Req *> reqs;
  std::vector<uint64_t> first;  // first chunk of each request (+ total)
  cudaStream_t st = nullptr;
  cudaEvent_t ev = nullptr;
  uint32_t slot0 = 0, nslot = 0;
  int phase = kRun;
  std::vector<void *> bufs;  // device allocations (stream-ordered)
  uint64_t bytes = 0;        // device buffer bytes charged to the budget
  std::vector<ChunkTask> tasks;  // in chunk order (not the launch order)
  uint8_t *d_in = nullptr, *d_scratch = nullptr, *d_out = nullptr, *d_image = nullptr;
  uint64_t *d_results = nullptr;
  uint32_t *d_status = nullptr, *d_queue = nullptr;  // d_queue[1]: tail-task counter
  TailTask *d_tails = nullptr;                        // compress: stale tails for the tail pass
  ModelInit *d_init = nullptr;
  ChunkTask *d_tasks = nullptr;
  uint64_t *h_lens = nullptr;  // pinned
  uint32_t *h_status = nullptr;
  std::vector<uint64_t> at_in, at_out;
  std::vector<uint64_t> redo;
  ModelInit init{};
  std::vector<uint8_t> image;
};

}  // namespace

struct cucm_server {
  int device = 0;
  int sm_count = 0;
  cucm_tuning tuning{};
  uint64_t budget = 0;       // device bytes for slots + buffers
  uint64_t buf_limit = 0;    // of which buffers
  uint64_t buf_used = 0;
  uint8_t *slots = nullptr;
  uint32_t nslots = 0;
  std::vector<uint8_t> slot_used;
  std::vector<cudaStream_t> idle_streams;
  std::vector<std::pair<void *, size_t>> pinned;  // idle pinned host blocks (never freed while serving)
  std::unordered_map<void *, size_t> pinned_sizes;
  cudaMemPool_t pool = nullptr;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Req *> queue;
  std::unordered_map<uint64_t, std::unique_ptr<Req>> reqs;
  std::vector<std::unique_ptr<Launch>> inflight;
  uint64_t next_id = 1;
  uint32_t max_queue = 1u << 16;
  bool stop = false;
  std::thread thr;
  // totals
  uint64_t completed = 0, bytes_in = 0, bytes_out = 0, launches = 0;
  int fatal = 0;
};

namespace {

#define SCK(call)                             \
  do {                                        \
    cudaError_t e_ = (call);                  \
    if (e_ != cudaSuccess) return CUCM_ECUDA; \
  } while (0)

// Prepare a request on the scheduler thread: parse / build the header and
// count its chunks.  Returns a status for the request.
int prepare(Req *r) {
  r->prepared = true;
  if (r->op == CUCM_OP_COMPRESS) {
    int rc = check_params(&r->p, r->n);
    if (rc) return rc;
    if (r->p.fixed_model) return CUCM_EINVAL;  // the serving loop codes the adaptive streams
    rc = make_header(r->in, r->n, &r->p, r->hdr, r->hm);
    if (rc) return rc;
    r->unit = r->p.unit;
    r->cs = r->p.chunksize;
    r->body_off = r->p.prelearn;
    r->body_n = r->n - r->p.prelearn;
    r->nchunks = (r->body_n + r->cs - 1) / r->cs;
    return CUCM_OK;
  }
  int rc = parse_header(r->in, r->n, r->ph);
  if (rc) return rc;
  if (r->ph.fixed) return CUCM_EINVAL;
  r->out_n = r->ph.total;
  if (r->ph.total > r->cap || (!r->out && r->ph.total)) return CUCM_ENOSPC;
  r->unit = r->ph.unit;
  r->cs = r->ph.cs;
  r->body_off = r->ph.body_off();
  r->body_n = r->n - r->body_off;
  r->out_body = r->ph.total - r->ph.prelearn;
  r->nchunks = (r->out_body + r->cs - 1) / r->cs;
  rc = parse_batches(r->in + r->body_off, r->body_n, r->nchunks, r->ph.batch, true, r->off, r->len, r->ph.wide);
  if (rc) return rc;
  if (r->ph.prelearn) {
    r->hm.reset(new HostModel());
    r->pre.resize(r->ph.prelearn);
    if (r->ph.coded)
      r->hm->prelearn_decode(r->in + r->ph.hdr, r->ph.pl_len, r->pre.data(), r->ph.prelearn);
    else {
      std::memcpy(r->pre.data(), r->in + r->ph.hdr, r->ph.prelearn);
      r->hm->prelearn_train(r->pre.data(), r->ph.prelearn);
    }
  }
  return CUCM_OK;
}

// Device buffer bytes a request needs while it runs.
uint64_t req_bytes(const Req *r) {
  const uint64_t pad = 256;
  if (r->op == CUCM_OP_COMPRESS)  // input, scratch, packed output, tasks, tail tasks
    return r->body_n + pad +
           r->nchunks * (2 * scratch_cap(r->cs) + sizeof(ChunkTask) + sizeof(PackEntry) + sizeof(TailTask) + 24) +
           4096;
  return r->body_n + pad + r->out_body + pad + r->nchunks * (sizeof(ChunkTask) + 16);
}

// Largest free run of slots, capped at `want`; returns its start and length.
uint32_t take_slots(cucm_server *s, uint32_t want, uint32_t *start) {
  uint32_t best = 0, best_at = 0, run = 0;
  for (uint32_t i = 0; i <= s->nslots; i++) {
    if (i < s->nslots && !s->slot_used[i]) {
      run++;
      if (run >= want) {
        best = want;
        best_at = i + 1 - want;
        break;
      }
    } else {
      if (run > best) {
        best = run;
        best_at = i - run;
      }
      run = 0;
    }
  }
  if (best > want) best = want;
  for (uint32_t i = 0; i < best; i++) s->slot_used[best_at + i] = 1;
  *start = best_at;
  return best;
}

// Pinned host blocks are kept and reused: allocating or freeing pinned
// memory can wait for the whole device, which would stall every launch.
void *pinned_get(cucm_server *s, size_t bytes) {
  for (size_t i = 0; i < s->pinned.size(); i++)
    if (s->pinned[i].second >= bytes) {
      void *p = s->pinned[i].first;
      s->pinned.erase(s->pinned.begin() + i);
      return p;
    }
  void *p = nullptr;
  size_t want = bytes < 4096 ? 4096 : bytes;
  if (cudaMallocHost(&p, want) != cudaSuccess) return nullptr;
  s->pinned_sizes[p] = want;
  return p;
}
void pinned_put(cucm_server *s, void *p) {
  if (p) s->pinned.push_back({p, s->pinned_sizes[p]});
}

void *dalloc(Launch *l, uint64_t bytes, cudaError_t *err) {
  void *p = nullptr;
  cudaError_t e = cudaMallocAsync(&p, bytes ? bytes : 16, l->st);
  if (e != cudaSuccess) {
    *err = e;
    return nullptr;
  }
  l->bufs.push_back(p);
  return p;
}

void finish_reqs(cucm_server *s, Launch *l, int status_all) {
  const double t = now_ms();
  std::lock_guard<std::mutex> g(s->mu);
  for (Req *r : l->reqs) {
    if (status_all && !r->status) r->status = status_all;
    r->done = true;
    r->t_done = t;
    s->completed++;
    s->bytes_in += r->n;
    s->bytes_out += r->status ? 0 : r->out_n;
  }
  s->cv_done.notify_all();
}

// Queue the final steps of a launch: clear its slots, then the event.
int close_launch(cucm_server *s, Launch *l) {
  SCK(cudaMemsetAsync(s->slots + (size_t)l->slot0 * kSlotTableBytes, 0, (size_t)l->nslot * kSlotTableBytes, l->st));
  SCK(cudaEventRecord(l->ev, l->st));
  l->phase = kFinish;
  return CUCM_OK;
}

int run_tasks(cucm_server *s, Launch *l, const std::vector<ChunkTask> &tasks) {
  EngineConfig cfg;
  cfg.spec_bits = s->tuning.spec_bits > 0 ? s->tuning.spec_bits : 4;
  cfg.generic = s->tuning.kernel == 1;
  cfg.sm_count = s->sm_count;
  cfg.dec_pairs = s->tuning.dec_pairs;
  cfg.dec_tables = s->tuning.dec_tables;
  cfg.cmp_ctas = s->tuning.cmp_ctas;
  cfg.spin_limit = s->tuning.dec_spin_limit;
  std::vector<ChunkTask> order = tasks;
  const bool dec = l->op == CUCM_OP_DECOMPRESS;
  std::stable_sort(order.begin(), order.end(), [&](const ChunkTask &a, const ChunkTask &b) {
    uint64_t la = (dec ? a.out_cap : a.in_len) * 4 + a.cs;
    uint64_t lb = (dec ? b.out_cap : b.in_len) * 4 + b.cs;
    return la > lb;
  });
  SCK(cudaMemcpyAsync(l->d_tasks, order.data(), sizeof(ChunkTask) * order.size(), cudaMemcpyHostToDevice, l->st));
  SCK(cudaMemsetAsync(l->d_queue, 0, 2 * sizeof(uint32_t), l->st));
  SCK(cudaMemsetAsync(l->d_status, 0, sizeof(uint32_t), l->st));
  const uint32_t grid = std::min<uint32_t>(l->nslot, (uint32_t)order.size());
  uint8_t *slots = s->slots + (size_t)l->slot0 * kSlotTableBytes;
  const uint8_t *img = l->model ? l->d_image : nullptr;
  cudaError_t e = dec ? launch_decompress(l->d_tasks, (uint32_t)order.size(), slots, grid, img, l->d_init, l->d_queue,
                                          l->d_status, cfg, l->st, (int)l->unit)
                      : launch_compress(l->d_tasks, (uint32_t)order.size(), slots, grid, img, l->d_init, l->d_queue,
                                        l->d_status, cfg, l->st, (int)l->unit, l->d_tails, l->d_queue + 1);
  SCK(e);
  s->launches++;
  return CUCM_OK;
}

// Start a launch for `grp` (prepared requests of one kind) on `nslot` slots.
int start_launch_in(cucm_server *s, Launch *l, std::vector<Req *> &grp, uint32_t slot0, uint32_t nslot,
                    uint64_t bytes) {
  l->op = grp[0]->op;
  l->unit = grp[0]->unit;
  l->model = grp[0]->hm != nullptr;
  l->reqs = grp;
  l->slot0 = slot0;
  l->nslot = nslot;
  l->bytes = bytes;
  if (!s->idle_streams.empty()) {
    l->st = s->idle_streams.back();
    s->idle_streams.pop_back();
  } else {
    SCK(cudaStreamCreateWithFlags(&l->st, cudaStreamNonBlocking));
  }
  SCK(cudaEventCreateWithFlags(&l->ev, cudaEventDisableTiming));
  const double t = now_ms();
  for (Req *r : grp) r->t_admit = t;
  l->first.assign(1, 0);
  for (Req *r : grp) l->first.push_back(l->first.back() + r->nchunks);
  const uint64_t nchunks = l->first.back();
  cudaError_t err = cudaSuccess;
  // model
  if (l->model) {
    grp[0]->hm->to_device(l->image, l->init);
  } else {
    for (int o = 0; o < kOrders; o++)
      for (int i = 0; i < 256; i++) l->init.statep[o][i] = 1u << 31;
    std::memset(l->init.w, 0, sizeof l->init.w);
  }
  l->d_init = (ModelInit *)dalloc(l, sizeof(ModelInit), &err);
  l->d_tasks = (ChunkTask *)dalloc(l, sizeof(ChunkTask) * std::max<uint64_t>(nchunks, 1), &err);
  l->d_queue = (uint32_t *)dalloc(l, 16, &err);
  l->d_status = (uint32_t *)dalloc(l, 16, &err);
  if (l->model) l->d_image = (uint8_t *)dalloc(l, kSlotTableBytes, &err);
  if (err != cudaSuccess) return CUCM_ENOMEM;
  SCK(cudaMemcpyAsync(l->d_init, &l->init, sizeof(ModelInit), cudaMemcpyHostToDevice, l->st));
  if (l->model) {
    SCK(cudaMemcpyAsync(l->d_image, l->image.data(), kSlotTableBytes, cudaMemcpyHostToDevice, l->st));
    // the launch's slots start from the prelearned tables
    for (uint32_t i = 0; i < nslot; i++)
      SCK(cudaMemcpyAsync(s->slots + (size_t)(slot0 + i) * kSlotTableBytes, l->d_image, kSlotTableBytes,
                          cudaMemcpyDeviceToDevice, l->st));
  }
  uint64_t in_tot = 0, out_tot = 0;
  for (Req *r : grp) {
    l->at_in.push_back(in_tot);
    in_tot += (r->body_n + 15) & ~15ull;
    l->at_out.push_back(out_tot);
    out_tot += l->op == CUCM_OP_COMPRESS ? 0 : ((r->out_body + 15) & ~15ull);
  }
  uint64_t smax = 0;
  for (Req *r : grp) smax = std::max(smax, scratch_cap(r->cs));
  l->d_in = (uint8_t *)dalloc(l, in_tot, &err);
  if (l->op == CUCM_OP_COMPRESS) {
    l->d_scratch = (uint8_t *)dalloc(l, nchunks * smax + 16, &err);
    l->d_tails = (TailTask *)dalloc(l, sizeof(TailTask) * std::max<uint64_t>(nchunks, 1), &err);
    l->d_results = (uint64_t *)dalloc(l, 8 * std::max<uint64_t>(nchunks, 1), &err);
  } else {
    l->d_out = (uint8_t *)dalloc(l, out_tot, &err);
  }
  if (err != cudaSuccess) return CUCM_ENOMEM;
  l->h_lens = (uint64_t *)pinned_get(s, 8 * std::max<uint64_t>(nchunks, 1));
  l->h_status = (uint32_t *)pinned_get(s, 16);
  if (!l->h_lens || !l->h_status) return CUCM_ENOMEM;
  // inputs
  for (size_t j = 0; j < grp.size(); j++) {
    Req *r = grp[j];
    if (r->body_n)
      SCK(cudaMemcpyAsync(l->d_in + l->at_in[j], r->in + r->body_off, r->body_n, cudaMemcpyHostToDevice, l->st));
  }
  // tasks in chunk order
  l->tasks.resize(nchunks);
  for (size_t j = 0; j < grp.size(); j++) {
    Req *r = grp[j];
    for (uint64_t k = 0; k < r->nchunks; k++) {
      ChunkTask &t = l->tasks[l->first[j] + k];
      t.cs = (uint32_t)r->cs;
      t.unit = r->unit;
      if (l->op == CUCM_OP_COMPRESS) {
        t.in = l->d_in + l->at_in[j] + k * r->cs;
        t.in_len = std::min<uint64_t>(r->cs, r->body_n - k * r->cs);
        t.out = l->d_scratch + (l->first[j] + k) * smax;
        t.out_cap = scratch_cap(r->cs);
        t.result = l->d_results + l->first[j] + k;
      } else {
        t.in = l->d_in + l->at_in[j] + r->off[k];
        t.in_len = r->len[k];
        t.out = l->d_out + l->at_out[j] + k * r->cs;
        t.out_cap = std::min<uint64_t>(r->cs, r->out_body - k * r->cs);
        t.result = nullptr;
      }
    }
  }
  int rc = CUCM_OK;
  if (nchunks) rc = run_tasks(s, l, l->tasks);
  if (rc) return rc;
  SCK(cudaMemcpyAsync(l->h_status, l->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, l->st));
  if (l->op == CUCM_OP_COMPRESS && nchunks)
    SCK(cudaMemcpyAsync(l->h_lens, l->d_results, 8 * nchunks, cudaMemcpyDeviceToHost, l->st));
  SCK(cudaEventRecord(l->ev, l->st));
  l->phase = kRun;
  return CUCM_OK;
}

// Release what a launch holds once its stream has drained: buffers, pinned
// memory, event, stream, slots (cleared again when the launch failed half
// way) and its share of the buffer budget.
void retire(cucm_server *s, Launch *l, bool clear_slots) {
  if (l->st) {
    if (clear_slots && l->nslot)
      cudaMemsetAsync(s->slots + (size_t)l->slot0 * kSlotTableBytes, 0, (size_t)l->nslot * kSlotTableBytes, l->st);
    for (void *p : l->bufs) cudaFreeAsync(p, l->st);
    cudaStreamSynchronize(l->st);
    s->idle_streams.push_back(l->st);
  }
  l->bufs.clear();
  for (uint32_t i = 0; i < l->nslot; i++) s->slot_used[l->slot0 + i] = 0;
  s->buf_used -= l->bytes;
  pinned_put(s, l->h_lens);
  pinned_put(s, l->h_status);
  l->h_lens = nullptr;
  l->h_status = nullptr;
  if (l->ev) cudaEventDestroy(l->ev);
}

int start_launch(cucm_server *s, std::vector<Req *> &grp, uint32_t slot0, uint32_t nslot, uint64_t bytes) {
  std::unique_ptr<Launch> L(new Launch());
  int rc = start_launch_in(s, L.get(), grp, slot0, nslot, bytes);
  if (rc) {
    retire(s, L.get(), true);
    finish_reqs(s, L.get(), rc);
    return rc;
  }
  std::lock_guard<std::mutex> g(s->mu);
  s->inflight.push_back(std::move(L));
  return CUCM_OK;
}

// Decompress launch whose kernel is done: outputs back to the callers.
int after_decode(cucm_server *s, Launch *l) {
  if (*l->h_status & kDevBadTask) return CUCM_EFORMAT;
  if (*l->h_status & kDevTimeout) return CUCM_ETIMEOUT;
  for (size_t j = 0; j < l->reqs.size(); j++) {
    Req *r = l->reqs[j];
    if (r->out_body)
      SCK(cudaMemcpyAsync(r->out + r->ph.prelearn, l->d_out + l->at_out[j], r->out_body, cudaMemcpyDeviceToHost,
                          l->st));
    if (r->ph.prelearn) std::memcpy(r->out, r->pre.data(), r->ph.prelearn);
  }
  return close_launch(s, l);
}

// Compress launch whose payload lengths are back: re-code overflowed chunks,
// or lay the containers out, pack and copy them back.
int after_encode(cucm_server *s, Launch *l) {
  const uint64_t nchunks = l->first.back();
  if (*l->h_status & kDevBadTask) return CUCM_EINVAL;
  if (l->phase == kRun) {
    for (uint64_t k = 0; k < nchunks; k++)
      if (l->h_lens[k] > l->tasks[k].out_cap) l->redo.push_back(k);
    if (!l->redo.empty()) {
      // slots are dirty after the first run; clear them, re-code with the hard bound
      SCK(cudaMemsetAsync(s->slots + (size_t)l->slot0 * kSlotTableBytes, 0, (size_t)l->nslot * kSlotTableBytes,
                          l->st));
      uint64_t tot = 0;
      for (uint64_t k : l->redo) tot += hard_cap(l->tasks[k].cs);
      cudaError_t err = cudaSuccess;
      uint8_t *big = (uint8_t *)dalloc(l, tot, &err);
      if (err != cudaSuccess) return CUCM_ENOMEM;
      std::vector<ChunkTask> rt;
      uint64_t at = 0;
      for (uint64_t k : l->redo) {
        ChunkTask t = l->tasks[k];
        t.out = big + at;
        t.out_cap = hard_cap(t.cs);
        at += t.out_cap;
        l->tasks[k] = t;
        rt.push_back(t);
      }
      int rc = run_tasks(s, l, rt);
      if (rc) return rc;
      SCK(cudaMemcpyAsync(l->h_lens, l->d_results, 8 * nchunks, cudaMemcpyDeviceToHost, l->st));
      SCK(cudaEventRecord(l->ev, l->st));
      l->phase = kRedo;
      return CUCM_OK;
    }
  }
  for (uint64_t k = 0; k < nchunks; k++)
    if (l->h_lens[k] > l->tasks[k].out_cap) return CUCM_ECUDA;
  // layout
  std::vector<const uint8_t *> src(nchunks);
  for (uint64_t k = 0; k < nchunks; k++) src[k] = l->tasks[k].out;
  std::vector<uint64_t> body(l->reqs.size()), at(l->reqs.size());
  uint64_t tot = 0;
  for (size_t j = 0; j < l->reqs.size(); j++) {
    Req *r = l->reqs[j];
    bool overflow = false;
    body[j] = layout_chunks(l->h_lens + l->first[j], src.data() + l->first[j], r->nchunks, r->p.batch, true, nullptr,
                            nullptr, wide_format(&r->p, r->n), &overflow);
    r->out_n = r->hdr.size() + body[j];
    if (overflow) r->status = CUCM_EINVAL;  // a batch past 4 GiB needs the 64-bit container
    else if (r->out_n > r->cap) r->status = CUCM_ENOSPC;
    at[j] = tot;
    tot += (body[j] + 15) & ~15ull;
  }
  cudaError_t err = cudaSuccess;
  uint8_t *d_out = (uint8_t *)dalloc(l, tot, &err);
  if (err != cudaSuccess) return CUCM_ENOMEM;
  std::vector<PackEntry> pe;
  for (size_t j = 0; j < l->reqs.size(); j++) {
    Req *r = l->reqs[j];
    if (r->status) continue;
    layout_chunks(l->h_lens + l->first[j], src.data() + l->first[j], r->nchunks, r->p.batch, true, d_out + at[j],
                  &pe, wide_format(&r->p, r->n));
  }
  if (!pe.empty()) {
    PackEntry *d_pe = (PackEntry *)dalloc(l, sizeof(PackEntry) * pe.size(), &err);
    if (err != cudaSuccess) return CUCM_ENOMEM;
    SCK(cudaMemcpyAsync(d_pe, pe.data(), sizeof(PackEntry) * pe.size(), cudaMemcpyHostToDevice, l->st));
    pack_kernel<<<(unsigned)pe.size(), 256, 0, l->st>>>(d_pe, (uint32_t)pe.size());
    SCK(cudaGetLastError());
  }
  for (size_t j = 0; j < l->reqs.size(); j++) {
    Req *r = l->reqs[j];
    if (r->status) continue;
    std::memcpy(r->out, r->hdr.data(), r->hdr.size());
    if (body[j])
      SCK(cudaMemcpyAsync(r->out + r->hdr.size(), d_out + at[j], body[j], cudaMemcpyDeviceToHost, l->st));
  }
  return close_launch(s, l);
}

// One pass over the in-flight launches: advance those whose event passed.
void progress(cucm_server *s) {
  for (size_t i = 0; i < s->inflight.size();) {
    Launch *l = s->inflight[i].get();
    const cudaError_t q = cudaEventQuery(l->ev);
    if (q == cudaErrorNotReady) {
      i++;
      continue;
    }
    int rc = q == cudaSuccess ? CUCM_OK : CUCM_ECUDA;
    if (!rc && l->phase != kFinish) {
      rc = l->op == CUCM_OP_COMPRESS ? after_encode(s, l) : after_decode(s, l);
      if (!rc) {
        i++;  // a new step is queued behind a new event
        continue;
      }
    }
    retire(s, l, rc != CUCM_OK);
    finish_reqs(s, l, rc);
    std::lock_guard<std::mutex> g(s->mu);
    s->inflight.erase(s->inflight.begin() + i);
  }
}

// Admit queued requests while slots and buffer memory allow.
void admit(cucm_server *s) {
  for (;;) {
    std::vector<Req *> cand;
    {
      std::lock_guard<std::mutex> g(s->mu);
      if (s->queue.empty()) return;
      cand.assign(s->queue.begin(), s->queue.end());
    }
    // prepare (host parsing / headers), failing requests finish at once
    std::vector<Req *> bad;
    for (Req *r : cand) {
      if (r->prepared) continue;
      r->status = prepare(r);
      // a request whose buffers alone exceed the buffer budget can never be
      // admitted within it
      if (!r->status && req_bytes(r) > s->buf_limit) r->status = CUCM_ENOMEM;
      if (r->status) bad.push_back(r);
    }
    if (!bad.empty()) {
      std::lock_guard<std::mutex> g(s->mu);
      const double t = now_ms();
      for (Req *r : bad) {
        r->done = true;
        r->t_done = t;
        s->completed++;
        s->queue.erase(std::find(s->queue.begin(), s->queue.end(), r));
      }
      s->cv_done.notify_all();
      continue;
    }
    // the head of the queue and every later request of its kind that fits;
    // other kinds wait for the next launch
    Req *h = cand[0];
    std::vector<Req *> grp{h};
    uint64_t need_slots = h->nchunks, bytes = req_bytes(h);
    if (!h->hm) {
      for (size_t j = 1; j < cand.size(); j++) {
        Req *r = cand[j];
        if (r->op != h->op || r->unit != h->unit || r->hm) continue;
        const uint64_t b = req_bytes(r);
        if (s->buf_used + bytes + b > s->buf_limit) break;
        grp.push_back(r);
        need_slots += r->nchunks;
        bytes += b;
      }
    }
    if (s->buf_used + bytes > s->buf_limit && !s->inflight.empty()) return;  // wait for memory
    uint32_t want = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(need_slots, 1), s->nslots);
    uint32_t slot0 = 0;
    const uint32_t got = take_slots(s, want, &slot0);
    if (got == 0) return;
    // a request needs at least one slot; with fewer slots than chunks the
    // persistent launch simply works through the queue
    s->buf_used += bytes;
    {
      std::lock_guard<std::mutex> g(s->mu);
      for (Req *r : grp) s->queue.erase(std::find(s->queue.begin(), s->queue.end(), r));
    }
    const int rc = start_launch(s, grp, slot0, got, bytes);
    if (rc == CUCM_ECUDA) s->fatal = rc;
  }
}

void scheduler(cucm_server *s) {
  cudaSetDevice(s->device);
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(s->mu);
      if (s->stop && s->queue.empty() && s->inflight.empty()) break;
      if (s->queue.empty() && s->inflight.empty())
        s->cv_work.wait_for(lk, std::chrono::milliseconds(50));
    }
    progress(s);
    admit(s);
    bool busy;
    {
      std::lock_guard<std::mutex> g(s->mu);
      busy = !s->inflight.empty();
    }
    if (busy) std::this_thread::sleep_for(std::chrono::microseconds(100));
  }
}

}  // namespace

extern "C" {

int cucm_server_create(int device, uint64_t hbm_budget, const cucm_tuning *tuning, cucm_server **out) {
  if (!out) return CUCM_EINVAL;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return CUCM_ENODEV;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) return CUCM_ENODEV;
  if (cudaSetDevice(device) != cudaSuccess) return CUCM_ENODEV;
  std::unique_ptr<cucm_server> s(new cucm_server());
  s->device = device;
  s->sm_count = prop.multiProcessorCount;
  if (tuning) s->tuning = *tuning;
  size_t freeb = 0, total = 0;
  cudaMemGetInfo(&freeb, &total);
  uint64_t budget = hbm_budget ? hbm_budget : (uint64_t)(0.9 * (double)freeb);
  if (budget > (uint64_t)(0.95 * (double)freeb)) budget = (uint64_t)(0.95 * (double)freeb);
  s->budget = budget;
  // a sixth of the budget (at least 2 GiB) for buffers, the rest for slots
  uint64_t bufs = std::max<uint64_t>(budget / 6, 2ull << 30);
  if (bufs >= budget) return CUCM_ENOMEM;
  uint64_t ns = (budget - bufs) / kSlotTableBytes;
  if (s->tuning.max_slots > 0) ns = std::min<uint64_t>(ns, (uint64_t)s->tuning.max_slots);
  if (ns == 0) return CUCM_ENOMEM;
  s->nslots = (uint32_t)ns;
  s->buf_limit = budget - ns * kSlotTableBytes;
  if (cudaMalloc(&s->slots, ns * kSlotTableBytes) != cudaSuccess) return CUCM_ENOMEM;
  if (cudaMemset(s->slots, 0, ns * kSlotTableBytes) != cudaSuccess) return CUCM_ECUDA;
  s->slot_used.assign(ns, 0);
  if (upload_tables() != cudaSuccess) return CUCM_ECUDA;
  // keep freed buffer memory in the pool instead of returning it to the driver
  if (cudaDeviceGetDefaultMemPool(&s->pool, device) == cudaSuccess) {
    uint64_t thr = s->buf_limit;
    cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return CUCM_ECUDA;
  cucm_server *raw = s.release();
  raw->thr = std::thread(scheduler, raw);
  *out = raw;
  return CUCM_OK;
}

int cucm_server_destroy(cucm_server *s) {
  if (!s) return CUCM_EINVAL;
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->thr.joinable()) s->thr.join();
  cudaSetDevice(s->device);
  for (cudaStream_t st : s->idle_streams) cudaStreamDestroy(st);
  for (auto &kv : s->pinned_sizes) cudaFreeHost(kv.first);
  cudaFree(s->slots);
  delete s;
  return CUCM_OK;
}

int cucm_serve_submit(cucm_server *s, int op, const uint8_t *in, uint64_t n, const cucm_params *p, uint8_t *out,
                      uint64_t cap, uint64_t *id) {
  if (!s || !id || (!in && n) || (op != CUCM_OP_COMPRESS && op != CUCM_OP_DECOMPRESS)) return CUCM_EINVAL;
  if (op == CUCM_OP_COMPRESS && (!p || !out)) return CUCM_EINVAL;
  if (op == CUCM_OP_DECOMPRESS && !in) return CUCM_EINVAL;
  std::unique_ptr<Req> r(new Req());
  r->op = op;
  r->in = in;
  r->n = n;
  if (p) r->p = *p;
  r->out = out;
  r->cap = cap;
  r->t_submit = now_ms();
  {
    std::lock_guard<std::mutex> g(s->mu);
    if (s->stop) return CUCM_EINVAL;
    if (s->fatal) return s->fatal;
    if (s->queue.size() >= s->max_queue) return CUCM_EBUSY;
    r->id = s->next_id++;
    *id = r->id;
    s->queue.push_back(r.get());
    s->reqs[r->id] = std::move(r);
  }
  s->cv_work.notify_all();
  return CUCM_OK;
}

int cucm_serve_poll(cucm_server *s, uint64_t id, int timeout_ms, int *status, uint64_t *out_n, double *latency_ms) {
  if (!s) return CUCM_EINVAL;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return CUCM_ENOTFOUND;
  Req *r = it->second.get();
  if (!r->done && timeout_ms != 0) {
    auto pred = [&] { return r->done; };
    if (timeout_ms < 0)
      s->cv_done.wait(lk, pred);
    else
      s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred);
  }
  if (!r->done) return CUCM_PENDING;
  if (status) *status = r->status;
  if (out_n) *out_n = r->out_n;
  if (latency_ms) *latency_ms = r->t_done - r->t_submit;
  s->reqs.erase(it);
  return CUCM_OK;
}

int cucm_server_set_queue_limit(cucm_server *s, uint32_t limit) {
  if (!s) return CUCM_EINVAL;
  std::lock_guard<std::mutex> g(s->mu);
  s->max_queue = limit;
  return CUCM_OK;
}

int cucm_server_stats(cucm_server *s, cucm_server_info *info) {
  if (!s || !info) return CUCM_EINVAL;
  std::lock_guard<std::mutex> g(s->mu);
  info->slots = s->nslots;
  info->budget = s->budget;
  info->completed = s->completed;
  info->bytes_in = s->bytes_in;
  info->bytes_out = s->bytes_out;
  info->launches = s->launches;
  info->queued = s->queue.size();
  info->inflight = s->inflight.size();
  return CUCM_OK;
}

}  // extern "C"
