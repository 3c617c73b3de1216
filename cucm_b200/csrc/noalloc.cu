// noalloc.cu -- a compress entry point that allocates no memory.
//
// Some callers cannot allocate device memory at the moment they want to
// compress: plugins inside a host application whose memory manager owns
// every device allocation (a cudaMalloc of their own would bypass its
// accounting and can fail once the application has reserved the device), and
// latency-critical paths that cannot afford cudaMalloc's implicit device
// synchronisation.  cucm_compress_chunk_noalloc serves them: the caller
// passes device input and output buffers, and the one piece of scratch the
// coder needs -- the bit-history tables of one chunk -- lives in the
// file-scope array g_noalloc_slot below.
//
// Costs and rules of that array:
//   * It is kSlotTableBytes (192.06 MiB: orders 0 and 1 by context, orders
//     2..7 at 2^25 one-byte slots each) and belongs to this file's own
//     module.  Under lazy module loading (CUDA_MODULE_LOADING=LAZY, the CUDA
//     12 default) the module, and with it the array, is loaded on a device
//     only when this entry point first runs there; with
//     CUDA_MODULE_LOADING=EAGER every context that loads libcucm.so reserves
//     the 192.06 MiB at once.  Once loaded, a GPU holds it until the process
//     exits.
//   * One call codes one chunk: the array holds one chunk's tables, so input
//     longer than the chunk size is rejected (CUCM_EINVAL).
//   * Every call shares the array and it keeps the last call's contents; each
//     call clears the tables on the caller's stream before its kernel runs.
//     Calls that overlap on the GPU (different streams, no ordering between
//     them) race on the array and produce garbage.  Serialise them.
//   * The call is synchronous: it reads the payload length back and waits
//     for the caller's stream before it returns.
//   * The first call on a device does the set-up (symbol addresses, constant
//     tables, kernel attributes) with that device current; make that first
//     call before any stream capture begins.  A set-up that fails is tried
//     again by the next call, except on a device that is not an sm_100 part.
// The kernel is the pipelined compressor of engine_kernels.cu, instantiated
// again in this module.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/cucm.h"
#include "engine.cuh"
#include "model.cuh"
#include "tables.h"

namespace cucm {
namespace {

__device__ Tables g_tables;

#include "device_common.cuh"
#include "compress_fast.cuh"

}  // namespace
}  // namespace cucm

using namespace cucm;

// The scratch of the no-allocation path (see the file comment).
static __device__ __align__(256) uint8_t g_noalloc_slot[kSlotTableBytes];
static __device__ ModelInit g_noalloc_init;
static __device__ uint32_t g_noalloc_status;
static __device__ uint64_t g_noalloc_result;

namespace {

struct NoAllocDevice {
  bool ready = false;     // set-up finished and succeeded
  bool foreign = false;   // not an sm_100 device: never usable
  uint8_t *slot = nullptr;
  ModelInit *init = nullptr;
  uint32_t *status = nullptr;
  uint64_t *result = nullptr;
};

constexpr int kMaxDevices = 64;
NoAllocDevice g_dev[kMaxDevices];
std::mutex g_mu;

// Once per device, with that device current: device addresses of the
// file-scope scratch (the host-side names are stand-ins, not addresses),
// the constant tables, the zero model and the kernel's shared-memory limit.
// Only success is remembered, so a transient failure is retried next call.
int noalloc_setup(int dev, NoAllocDevice *&out) {
  std::lock_guard<std::mutex> g(g_mu);
  NoAllocDevice &d = g_dev[dev];
  out = &d;
  if (d.ready) return CUCM_OK;
  if (d.foreign) return CUCM_ENODEV;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return CUCM_ECUDA;
  if (prop.major != 10) {
    d.foreign = true;
    return CUCM_ENODEV;
  }
  if (cudaGetSymbolAddress((void **)&d.slot, g_noalloc_slot) != cudaSuccess) return CUCM_ECUDA;
  if (cudaGetSymbolAddress((void **)&d.init, g_noalloc_init) != cudaSuccess) return CUCM_ECUDA;
  if (cudaGetSymbolAddress((void **)&d.status, g_noalloc_status) != cudaSuccess) return CUCM_ECUDA;
  if (cudaGetSymbolAddress((void **)&d.result, g_noalloc_result) != cudaSuccess) return CUCM_ECUDA;
  Tables t;
  build_tables(t);
  if (cudaMemcpyToSymbol(g_tables, &t, sizeof t) != cudaSuccess) return CUCM_ECUDA;
  ModelInit zero;
  for (int o = 0; o < kOrders; o++)
    for (int s = 0; s < 256; s++) zero.statep[o][s] = 1u << 31;
  for (int i = 0; i < kMixCtx * kOrders; i++) zero.w[i] = 0;
  if (cudaMemcpyToSymbol(g_noalloc_init, &zero, sizeof zero) != cudaSuccess) return CUCM_ECUDA;
  const size_t smem = make_fast_layout(kFastMaxUnit).total;
  if (cudaFuncSetAttribute((const void *)compress_fast_single_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return CUCM_ECUDA;
  if (cudaFuncSetAttribute((const void *)compress_fast_single_kernel<16>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return CUCM_ECUDA;
  d.ready = true;
  return CUCM_OK;
}

}  // namespace

extern "C" int cucm_compress_chunk_noalloc(const uint8_t *d_in, uint64_t len, uint64_t chunksize, uint32_t unit,
                                           uint8_t *d_out, uint64_t cap, uint64_t *out_len, void *stream) {
  if (!d_in || !d_out || !out_len) return CUCM_EINVAL;
  if (chunksize == 0 || chunksize > 0xffffffffull) return CUCM_EINVAL;
  if (len == 0 || len > chunksize) return CUCM_EINVAL;  // one chunk per call: the scratch holds one chunk's tables
  if (unit < 32 || unit > (uint32_t)kFastMaxUnit || unit % 32) return CUCM_EINVAL;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return CUCM_ENODEV;
  NoAllocDevice *d = nullptr;
  int rc = noalloc_setup(dev, d);
  if (rc) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  // The tables start from the zero model; the previous call left its own.
  if (cudaMemsetAsync(d->slot, 0, kSlotTableBytes, st) != cudaSuccess) return CUCM_ECUDA;
  if (cudaMemsetAsync(d->status, 0, sizeof(uint32_t), st) != cudaSuccess) return CUCM_ECUDA;
  ChunkTask t;
  t.in = d_in;
  t.out = d_out;
  t.in_len = len;
  t.out_cap = cap;
  t.cs = (uint32_t)chunksize;
  t.unit = unit;
  t.result = d->result;
  const size_t smem = make_fast_layout((int)unit).total;
  if (unit <= 128)
    compress_fast_single_kernel<8><<<1, kFastThreads, smem, st>>>(t, d->slot, d->init, d->status);
  else
    compress_fast_single_kernel<16><<<1, kFastThreads, smem, st>>>(t, d->slot, d->init, d->status);
  if (cudaGetLastError() != cudaSuccess) return CUCM_ECUDA;
  uint64_t got = 0;
  uint32_t status = 0;
  if (cudaMemcpyAsync(&got, d->result, sizeof got, cudaMemcpyDeviceToHost, st) != cudaSuccess) return CUCM_ECUDA;
  if (cudaMemcpyAsync(&status, d->status, sizeof status, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return CUCM_ECUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return CUCM_ECUDA;
  *out_len = got;
  if (status & kDevBadTask) return CUCM_EINVAL;
  if (status & ~(uint32_t)kDevOverflow) return CUCM_ECUDA;  // any other device status is an error
  if (got > cap) return CUCM_ENOSPC;
  return CUCM_OK;
}
