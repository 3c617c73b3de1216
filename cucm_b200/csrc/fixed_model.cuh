// fixed_model.cuh -- the fixed-model variant (the paper's section 4.5).
//
// Included by engine_kernels.cu (shares its tables).
//
// The paper discusses, and measures, keeping CuCM's model fixed after the
// prelearn pass: no StateMap or Mixer update while the data is coded.  The
// reference ships no code for it; this build defines its stream (container
// flag bit 1): every data bit of a chunk is predicted by the prelearned
// model as the prelearn pass predicts (keys over the chunk's own history,
// StateMaps, Mixer -- cucm_compress_v2.cu:930-955) and coded with the
// reference's binary coder; only the data bits are coded (no stale tail),
// then the flush byte.
//
// Nothing is written during coding, so one copy of the model serves every
// chunk: the slot image (192 MiB, read through the read-only cache and L2),
// and per CTA in shared memory the stretched probabilities of the 256
// states of each order and the 640 mixer weights.  That makes the variant
// two kernels instead of a pipeline:
//
//   fixed_prob_kernel   one thread per input byte computes its 8 bits'
//                       coder inputs (pr << 1 | y) -- every bit of every
//                       chunk in parallel -- into a u16 array;
//   fixed_coder_kernel  one thread per chunk runs the arithmetic coder over
//                       its chunk's array;
//
// and the decoder is one warp per chunk decoding a nibble per round over the
// 15-node speculation tree, the next round's gathers issued as soon as a
// round is decided.

constexpr int kFixedThreads = 256;

struct FixedSmem {
  int16_t spf[256 * kOrders];  // stretched statep of the model, [state][order]
  int32_t w[kMixCtx * kOrders];
  uint16_t squash[4096];
};

__device__ inline void fixed_load_model(FixedSmem *f, const ModelInit *init) {
  for (int i = threadIdx.x; i < 256 * kOrders; i += blockDim.x)
    f->spf[i] = g_tables.stretch[init->statep[i & 7][i >> 3] >> 20];
  for (int i = threadIdx.x; i < kMixCtx * kOrders; i += blockDim.x) f->w[i] = init->w[i];
  for (int i = threadIdx.x; i < 4096; i += blockDim.x) f->squash[i] = g_tables.squash[i];
}

// The state of one order's key in the read-only slot image.
__device__ __forceinline__ uint32_t fixed_state(const uint8_t *image, int o, uint32_t key) {
  return __ldg(image + table_offset(o) + key);
}

// Mixer output (Mixer::p, cucm_compress_v2.cu:636-644, then pr++ below 2048)
// for the stretched inputs of one bit.
__device__ __forceinline__ int fixed_mix(const FixedSmem *f, const int smp[kOrders], int c1) {
  int olen = 0;
CUCM_UNROLL
  for (int o = 0; o < kOrders; o++) olen += smp[o] != 1;
  const int cxt = olen + (c1 >> 5) * 10;
  long long sum = 0;
CUCM_UNROLL
  for (int o = 0; o < kOrders; o++) sum += (long long)f->w[cxt * kOrders + o] * smp[o];
  sum >>= 16;
  const int idx = sum < -2047 ? -2047 : (sum > 2048 ? 2048 : (int)sum);
  const int pr = f->squash[idx + 2047];
  return pr < 2048 ? pr + 1 : pr;
}

// Thread = (task, byte): each CTA pass covers 256 consecutive bytes of all
// the tasks' bytes laid end to end.  `first` holds each task's first index in
// that sequence (prefix sums of the chunk lengths), `total` its length.
__global__ void __launch_bounds__(kFixedThreads)
    fixed_prob_kernel(const FixedTask *tasks, const uint64_t *first, uint32_t ntasks, uint64_t total,
                      const uint8_t *image, const ModelInit *init) {
  __shared__ FixedSmem f;
  __shared__ uint32_t s_task;
  fixed_load_model(&f, init);
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < total; base += (uint64_t)gridDim.x * blockDim.x) {
    __syncthreads();
    if (threadIdx.x == 0) {  // the task holding byte `base`
      uint32_t lo = 0, hi = ntasks - 1;
      while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (first[mid] <= base) lo = mid; else hi = mid - 1;
      }
      s_task = lo;
    }
    __syncthreads();
    const uint64_t gi = base + threadIdx.x;
    if (gi >= total) continue;
    uint32_t ti = s_task;
    while (ti + 1 < ntasks && first[ti + 1] <= gi) ti++;
    const FixedTask &t = tasks[ti];
    const uint64_t q = gi - first[ti];
    const uint8_t *in = t.in;
    uint32_t hist[7];
CUCM_UNROLL
    for (int i = 0; i < 7; i++) hist[i] = q > (uint64_t)i ? __ldg(in + q - 1 - i) : 0u;
    const uint32_t cur = __ldg(in + q);
    uint16_t e[8];
CUCM_UNROLL
    for (int r = 0; r < 8; r++) {
      const uint32_t h0 = (1u << r) | (cur >> (8 - r));
      BitKeys kk;
      bit_keys(h0, hist, kk);
      int smp[kOrders];
CUCM_UNROLL
      for (int o = 0; o < kOrders; o++) smp[o] = f.spf[fixed_state(image, o, kk.k[o]) * kOrders + o];
      const int pr = fixed_mix(&f, smp, (int)hist[0]);
      e[r] = (uint16_t)((pr << 1) | ((cur >> (7 - r)) & 1u));
    }
    uint4 v;
    v.x = e[0] | ((uint32_t)e[1] << 16);
    v.y = e[2] | ((uint32_t)e[3] << 16);
    v.z = e[4] | ((uint32_t)e[5] << 16);
    v.w = e[6] | ((uint32_t)e[7] << 16);
    *reinterpret_cast<uint4 *>(t.prm + 8 * q) = v;
  }
}

// Thread = task: the binary coder over the chunk's coder inputs, eight per
// load (coder_step's arithmetic), bytes straight to the payload, then the
// flush byte (cucm_compress_v2.cu:902) and the payload length.
__global__ void __launch_bounds__(128) fixed_coder_kernel(const FixedTask *tasks, uint32_t ntasks, uint32_t *status) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ntasks) return;
  const FixedTask t = tasks[i];
  uint32_t x1 = 0, x2 = 0xffffffffu;
  uint64_t head = 0;
  const uint4 *src = reinterpret_cast<const uint4 *>(t.prm);
  const uint64_t n = t.in_len;
  // four bytes' inputs per group; the next group's loads are in flight
  // while the current one is coded
  uint4 nxt[4];
CUCM_UNROLL
  for (int b = 0; b < 4; b++) nxt[b] = (uint64_t)b < n ? __ldg(src + b) : make_uint4(0, 0, 0, 0);
  for (uint64_t q = 0; q < n; q += 4) {
    uint4 cur[4];
CUCM_UNROLL
    for (int b = 0; b < 4; b++) {
      cur[b] = nxt[b];
      nxt[b] = q + 4 + b < n ? __ldg(src + q + 4 + b) : make_uint4(0, 0, 0, 0);
    }
CUCM_UNROLL
    for (int b = 0; b < 4; b++) {
      if (q + b >= n) break;
      const uint32_t w4[4] = {cur[b].x, cur[b].y, cur[b].z, cur[b].w};
CUCM_UNROLL
      for (int h = 0; h < 8; h++) {
        const uint32_t e = (w4[h >> 1] >> (16 * (h & 1))) & 0xffffu;
        const uint32_t xm = x1 + __umulhi(x2 - x1, (e >> 1) << 20);
        if (e & 1) x2 = xm; else x1 = xm + 1;
        while ((x1 ^ x2) < 0x1000000u) {
          if (head < t.out_cap) t.out[head] = (uint8_t)(x2 >> 24);
          head++;
          x1 <<= 8;
          x2 = (x2 << 8) | 255u;
        }
      }
    }
  }
  if (head < t.out_cap) t.out[head] = (uint8_t)(x1 >> 24);
  head++;
  *t.result = head;
  if (head > t.out_cap) atomicOr(status, (uint32_t)kDevOverflow);
}

constexpr int kFixedDecWarps = 8;

// Warp = chunk (tasks handed out by a queue).  Lanes 0..14 are the nodes of
// the nibble's speculation tree (lanes 15..31 mirror them so every load stays
// uniform); each gathers its 8 states, mixes, and the warp decodes the 4
// bits uniformly (cucm_decompress_v2.cu:813-868's coder).  The window of the
// payload is staged per warp in shared memory.
__global__ void __launch_bounds__(kFixedDecWarps * 32)
    fixed_decode_kernel(const FixedTask *tasks, uint32_t ntasks, const uint8_t *image, const ModelInit *init,
                        uint32_t *queue) {
  __shared__ FixedSmem f;
  __shared__ __align__(16) uint8_t wins[kFixedDecWarps][kDecWin];
  fixed_load_model(&f, init);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint8_t *win = wins[warp];
  const int node = lane % kDecNodes;
  const int depth = 31 - __clz(node + 1);
  const uint32_t pbits = (uint32_t)(node + 1 - (1 << depth));
  for (;;) {
    uint32_t ti = 0;
    if (lane == 0) ti = atomicAdd(queue, 1u);
    ti = __shfl_sync(0xffffffffu, ti, 0);
    if (ti >= ntasks) break;
    const FixedTask t = tasks[ti];
    const uint8_t *pay = t.in;
    const uint64_t plen = t.in_len;
    long long wbase = dec_refill(win, pay, plen, 0, lane);
    uint32_t x1 = 0, x2 = 0xffffffffu, x = 0;
    uint64_t ioff = 0;
    for (int i = 0; i < 4; i++, ioff++) x = (x << 8) | (ioff < plen ? (uint32_t)win[(long long)ioff - wbase] : 255u);
    uint32_t hist[7] = {0, 0, 0, 0, 0, 0, 0};
    uint32_t cur = 0;
    int r = 0;
    uint32_t st[kOrders];
    auto gather = [&]() {
      const uint32_t h0 = (1u << (r + depth)) | (cur << depth) | pbits;
      BitKeys kk;
      bit_keys(h0, hist, kk);
CUCM_UNROLL
      for (int o = 0; o < kOrders; o++) st[o] = fixed_state(image, o, kk.k[o]);
    };
    const uint64_t rounds = 2 * t.out_cap;
    if (rounds) gather();
    for (uint64_t rd = 0; rd < rounds; rd++) {
      if ((long long)ioff + 16 > wbase + kDecWin) wbase = dec_refill(win, pay, plen, ioff, lane);
      int smp[kOrders];
CUCM_UNROLL
      for (int o = 0; o < kOrders; o++) smp[o] = f.spf[st[o] * kOrders + o];
      const uint32_t f_node = (uint32_t)fixed_mix(&f, smp, (int)hist[0]) << 20;
      int n = 0;
      uint32_t nib = 0;
      uint32_t fv = __shfl_sync(0xffffffffu, f_node, 0);
CUCM_UNROLL
      for (int i = 0; i < 4; i++) {
        uint32_t fa = 0, fb = 0;
        if (i < 3) {
          fa = __shfl_sync(0xffffffffu, f_node, 2 * n + 1);
          fb = __shfl_sync(0xffffffffu, f_node, 2 * n + 2);
        }
        const uint32_t xm = x1 + __umulhi(x2 - x1, fv);
        const int y = x <= xm;
        if (y) x2 = xm; else x1 = xm + 1;
        while ((x1 ^ x2) < 0x1000000u) {
          x1 <<= 8;
          x2 = (x2 << 8) | 255u;
          x = (x << 8) | (ioff < plen ? (uint32_t)win[(long long)ioff - wbase] : 255u);
          ioff++;
        }
        nib = (nib << 1) | (uint32_t)y;
        n = 2 * n + 1 + y;
        fv = y ? fb : fa;
      }
      cur = (cur << 4) | nib;
      r += 4;
      if (r == 8) {
        if (lane == 0) t.out[rd >> 1] = (uint8_t)cur;
CUCM_UNROLL
        for (int i = 6; i > 0; i--) hist[i] = hist[i - 1];
        hist[0] = cur;
        cur = 0;
        r = 0;
      }
      if (rd + 1 < rounds) gather();
    }
    __syncwarp();
  }
}
