// engine_kernels.cu -- the CuCM chunk coder as sm_100a kernels.
//
// One CTA owns one chunk at a time and walks it unit by unit with the
// reference's schedule (cucm_compress_v2.cu:1067-1090, decoder
// cucm_decompress_v2.cu:977-1032): every prediction of a unit reads the model
// as it was at the unit start; mixer deltas and StateMap updates are applied
// when the unit is done.  Instead of one launch per phase and a host round
// trip per unit, the whole chunk runs inside one CTA:
//
//   front phase (all warps): keys of every (bit, order), gathers of the
//       frozen bit-history states, stretch/mix/squash, mixer deltas;
//   chain (warp 0, lane = order): the serial StateMap update of the unit,
//       with same-slot updates inside the unit resolved through a per-order
//       shared-memory overlay (open addressing, slot -> live state);
//   coder (warp 1, lane 0): the 32-bit binary arithmetic coder, output
//       staged in a shared-memory ring and written out in 512-byte blocks;
//   write-back (all warps): the overlay's final states go to the slot tables
//       before the next unit gathers.
//
// A CTA takes chunks from a global queue (persistent form) until it is
// empty; the plain form launches one single-CTA grid per chunk.
#include <algorithm>
#include <cuda_runtime.h>

#include <cstdint>

#include "engine.cuh"
#include "model.cuh"
#include "tables.h"

namespace cucm {

namespace {

__device__ Tables g_tables;

#include "device_common.cuh"

struct Layout {
  int U, NB, logNB, stage;
  size_t off_tab, off_statep, off_w, off_key, off_okey, off_fs, off_ost, off_yb, off_prm, off_cxt,
      off_stage, off_misc, total;
};

__host__ __device__ inline Layout make_layout(int U, int extra_node_bytes) {
  Layout L;
  L.U = U;
  L.NB = next_pow2(2 * U);
  L.logNB = ilog2(L.NB);
  L.stage = next_pow2(4 * U + 1024);
  if (L.stage < kStageMin) L.stage = kStageMin;
  size_t o = 0;
  L.off_tab = o;     o += sizeof(Tables);
  L.off_statep = o;  o += sizeof(uint32_t) * kOrders * 256;
  L.off_w = o;       o += sizeof(int32_t) * kMixCtx * kOrders;
  L.off_key = o;     o += sizeof(uint32_t) * kOrders * U;
  L.off_okey = o;    o += sizeof(uint32_t) * kOrders * L.NB;
  L.off_fs = o;      o += (size_t)kOrders * U;
  L.off_ost = o;     o += (size_t)kOrders * L.NB;
  L.off_yb = o;      o += (size_t)U;
  L.off_prm = o;     o += sizeof(uint16_t) * U;
  L.off_cxt = o;     o += (size_t)U;
  o = (o + 15) & ~(size_t)15;
  L.off_stage = o;   o += (size_t)L.stage + (size_t)extra_node_bytes;
  L.off_misc = o;    o += 64;
  L.total = o;
  return L;
}

struct Smem {
  Tables *tab;
  uint32_t *statep;  // [8][256]
  int32_t *w;        // [80*8]
  uint32_t *key;     // [8][U]
  uint32_t *okey;    // [8][NB]   0 = empty, else key + 1
  uint8_t *fs;       // [8][U]    frozen (unit-start) state
  uint8_t *ost;      // [8][NB]   overlay live state
  uint8_t *yb;       // [U]
  uint16_t *prm;     // [U]       pr << 1 | y
  uint8_t *cxt;      // [U]
  uint8_t *stage;    // coder output ring (compress) / payload window + nodes (decompress)
  int *misc;
};

__device__ inline Smem carve(uint8_t *base, const Layout &L) {
  Smem s;
  s.tab = reinterpret_cast<Tables *>(base + L.off_tab);
  s.statep = reinterpret_cast<uint32_t *>(base + L.off_statep);
  s.w = reinterpret_cast<int32_t *>(base + L.off_w);
  s.key = reinterpret_cast<uint32_t *>(base + L.off_key);
  s.okey = reinterpret_cast<uint32_t *>(base + L.off_okey);
  s.fs = base + L.off_fs;
  s.ost = base + L.off_ost;
  s.yb = base + L.off_yb;
  s.prm = reinterpret_cast<uint16_t *>(base + L.off_prm);
  s.cxt = base + L.off_cxt;
  s.stage = base + L.off_stage;
  s.misc = reinterpret_cast<int *>(base + L.off_misc);
  return s;
}

__device__ inline void load_model(const Smem &s, const ModelInit *init, const Layout &L) {
  for (int i = threadIdx.x; i < kOrders * 256; i += blockDim.x) s.statep[i] = init->statep[i / 256][i % 256];
  for (int i = threadIdx.x; i < kMixCtx * kOrders; i += blockDim.x) s.w[i] = init->w[i];
  for (int i = threadIdx.x; i < kOrders * L.NB; i += blockDim.x) s.okey[i] = 0;
  for (int i = threadIdx.x; i < L.U; i += blockDim.x) s.prm[i] = 0;  // cucm_compress_v2.cu:1039-1040
}

// Predictions of the 8 orders from frozen states, stretched, and the mixer
// context (cucm_compress_v2.cu:770-784).
__device__ __forceinline__ int stretch_and_cxt(const Smem &s, const uint8_t st[kOrders], int c1, int smp[kOrders]) {
  int olen = 0;
#pragma unroll
  for (int o = 0; o < kOrders; o++) {
    uint32_t p = s.statep[o * 256 + st[o]] >> 20;
    smp[o] = s.tab->stretch[p];
    olen += (smp[o] != 1);
  }
  return olen + (c1 >> 5) * 10;
}

// Mixer deltas of one bit added to the weights (Mixer::update,
// cucm_compress_v2.cu:663-678).  Integer adds commute, so the order in which
// threads add is irrelevant.
__device__ __forceinline__ void mixer_train(int32_t *w, int cxt, const int smp[kOrders], int y, int pr) {
  int err = ((y << 12) - pr) * 7;
#pragma unroll
  for (int o = 0; o < kOrders; o++) {
    int d = (int)(((long long)err * smp[o]) >> 16);
    atomicAdd(&w[cxt * kOrders + o], d);
  }
}

// Serial StateMap update of one order over the unit's bits (lane = order).
// Reads the live state of each slot: the overlay holds slots already updated
// in this unit, anything else is the frozen state gathered at unit start.
__device__ inline void chain_order(const Smem &s, const Layout &L, int o, int n) {
  const uint32_t *key = s.key + o * L.U;
  const uint8_t *fs = s.fs + o * L.U;
  uint32_t *okey = s.okey + o * L.NB;
  uint8_t *ost = s.ost + o * L.NB;
  uint32_t *sp = s.statep + o * 256;
  const Tables *t = s.tab;
  for (int j = 0; j < n; j++) {
    uint32_t k = key[j];
    int y = s.yb[j];
    uint32_t b = bucket_of(k, L.logNB);
    int st;
    for (;;) {
      uint32_t kk = okey[b];
      if (kk == k + 1) {
        st = ost[b];
        break;
      }
      if (kk == 0) {
        st = fs[j];
        okey[b] = k + 1;
        break;
      }
      b = (b + 1) & (L.NB - 1);
    }
    uint32_t v = sp[st];
    sp[st] = statep_next(v, y, t->dt[v & 1023u]);
    ost[b] = t->nex[st][y];
  }
}

// Overlay -> slot tables, then clear the overlay.
__device__ inline void write_back(const Smem &s, const Layout &L, uint8_t *slot) {
  for (int i = threadIdx.x; i < kOrders * L.NB; i += blockDim.x) {
    uint32_t kk = s.okey[i];
    if (kk) {
      int o = i / L.NB;
      slot[table_offset(o) + (kk - 1)] = s.ost[i];
      s.okey[i] = 0;
    }
  }
}

__device__ inline void coder_run(Coder &c, const Smem &s, const Layout &L, int n) {
  coder_run_p(c, s.prm, s.stage, L.stage, n);
}
__device__ inline void coder_flush_blocks(Coder &c, const Smem &s, const Layout &L, uint8_t *out, uint64_t cap) {
  coder_flush_p(c, s.stage, L.stage, out, cap);
}
__device__ inline void coder_finish(Coder &c, const Smem &s, const Layout &L, uint8_t *out, uint64_t cap,
                                    uint64_t *result) {
  coder_finish_p(c, s.stage, L.stage, out, cap, result);
}

__device__ void compress_one(const ChunkTask &t, uint8_t *slot, const Smem &s, const Layout &L,
                             const ModelInit *init, uint32_t *status) {
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const uint64_t len = t.in_len < t.cs ? t.in_len : t.cs;
  const uint64_t total_bits = 8ull * t.cs;
  const uint64_t data_bits = 8ull * len;
  const int U = L.U;
  const uint8_t *in = t.in;

  load_model(s, init, L);
  Coder c{0u, 0xffffffffu, 0, 0};
  __syncthreads();

  uint64_t base = 0;
  for (; base < data_bits; base += U) {
    const int nvalid = (int)(data_bits - base < (uint64_t)U ? data_bits - base : (uint64_t)U);
    const int ncode = (int)(total_bits - base < (uint64_t)U ? total_bits - base : (uint64_t)U);

    // Phase 1: keys and frozen-state gathers (cudapredictUnit).
    for (int j = tid; j < nvalid; j += blockDim.x) {
      uint64_t b = base + j;
      uint64_t q = b >> 3;
      int r = (int)(b & 7);
      uint32_t cur = in[q];
      uint32_t h0 = (1u << r) | (cur >> (8 - r));
      uint32_t hist[7];
#pragma unroll
      for (int i = 0; i < 7; i++) hist[i] = q >= (uint64_t)(i + 1) ? in[q - 1 - i] : 0u;
      BitKeys k;
      bit_keys(h0, hist, k);
      uint8_t st[kOrders];
#pragma unroll
      for (int o = 0; o < kOrders; o++) st[o] = slot[table_offset(o) + k.k[o]];
#pragma unroll
      for (int o = 0; o < kOrders; o++) {
        s.key[o * U + j] = k.k[o];
        s.fs[o * U + j] = st[o];
      }
      s.yb[j] = (uint8_t)((cur >> (7 - r)) & 1u);
    }
    __syncthreads();

    // Phase 2: stretch, mixer context, mixer output (cudamixUnit).
    for (int j = tid; j < nvalid; j += blockDim.x) {
      uint64_t b = base + j;
      uint64_t q = b >> 3;
      uint8_t st[kOrders];
#pragma unroll
      for (int o = 0; o < kOrders; o++) st[o] = s.fs[o * U + j];
      int smp[kOrders];
      int c1 = q >= 1 ? in[q - 1] : 0;
      int cx = stretch_and_cxt(s, st, c1, smp);
      int pr = mix_pr(s.w, cx, smp, s.tab);
      s.prm[j] = (uint16_t)((pr << 1) | s.yb[j]);
      s.cxt[j] = (uint8_t)cx;
    }
    __syncthreads();

    // Phase 2b: mixer deltas (cudaupdateMixer); reads statep, so before the chain.
    for (int j = tid; j < nvalid; j += blockDim.x) {
      uint8_t st[kOrders];
#pragma unroll
      for (int o = 0; o < kOrders; o++) st[o] = s.fs[o * U + j];
      int smp[kOrders];
#pragma unroll
      for (int o = 0; o < kOrders; o++) smp[o] = s.tab->stretch[s.statep[o * 256 + st[o]] >> 20];
      mixer_train(s.w, s.cxt[j], smp, s.prm[j] & 1, s.prm[j] >> 1);
    }
    __syncthreads();

    // Phase 3: StateMap chain (warp 0) and coder (warp 1) side by side.
    if (warp == 0) {
      if (tid < kOrders) chain_order(s, L, tid, nvalid);
    } else if (warp == 1) {
      coder_run(c, s, L, ncode);
      coder_flush_blocks(c, s, L, t.out, t.out_cap);
    }
    __syncthreads();

    // Phase 4: write-back of the unit's final slot states.
    write_back(s, L, slot);
    __syncthreads();
  }

  // Past the input: the coder keeps coding the stale prm buffer up to the
  // chunk end (cucm_compress_v2.cu:850-852 check only the chunk bound).
  if (warp == 1) {
    for (; base < total_bits; base += U) {
      const int ncode = (int)(total_bits - base < (uint64_t)U ? total_bits - base : (uint64_t)U);
      coder_run(c, s, L, ncode);
      coder_flush_blocks(c, s, L, t.out, t.out_cap);
    }
    coder_finish(c, s, L, t.out, t.out_cap, t.result);
    if ((tid & 31) == 0 && c.head > t.out_cap) atomicOr(status, (uint32_t)kDevOverflow);
  }
  __syncthreads();
}

__global__ void __launch_bounds__(256) compress_kernel(const ChunkTask *tasks, uint32_t ntasks, uint8_t *slots,
                                                       const uint8_t *init_tables, const ModelInit *init,
                                                       uint32_t *queue, uint32_t *status, int unit) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  const Layout L = make_layout(unit, 0);
  const Smem s = carve(smem_raw, L);
  uint8_t *slot = slots + (size_t)blockIdx.x * kSlotTableBytes;
  copy_tables(&g_tables, s.tab);
  __shared__ uint32_t s_task;
  bool fresh = true;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_task = atomicAdd(queue, 1u);
    __syncthreads();
    const uint32_t ti = s_task;
    if (ti >= ntasks) break;
    const ChunkTask t = tasks[ti];
    if (t.unit != (uint32_t)unit || t.cs == 0) {
      if (threadIdx.x == 0) {
        atomicOr(status, (uint32_t)kDevBadTask);
        *t.result = ~0ull;
      }
      continue;
    }
    if (!fresh) {
      reset_slot(slot, init_tables);
      __syncthreads();
    }
    fresh = false;
    compress_one(t, slot, s, L, init, status);
  }
}

// ---------------------------------------------------------------------------
// Decompression.

// Payload window: bytes [win_base, win_base + kWin) of the chunk payload.
constexpr int kWin = 2048;
// Speculation-tree node arrays (up to 255 nodes), each 16-byte aligned.
constexpr size_t kNodeKeyBytes = sizeof(uint32_t) * kOrders * 255 + 16;  // 8176
constexpr size_t kNodePrBytes = sizeof(uint16_t) * 256;                  // 512
constexpr size_t kNodeFsBytes = kOrders * 255 + 8;                       // 2048
constexpr size_t kNodeCxtBytes = 256;
constexpr size_t kNodeBytes = kNodeKeyBytes + kNodePrBytes + kNodeFsBytes + kNodeCxtBytes;

struct DecState {
  uint32_t x1, x2, x;
  uint64_t ioff;      // next payload byte to shift in
  uint64_t pos;       // next bit to decode (chunk bit index)
  uint64_t hist;      // completed bytes, byte 0 = most recent
  uint32_t cur;       // bits of the current byte so far
  int r;              // number of bits in cur
};

// Node n of the speculation tree: prefix length l = floor(log2(n+1)), prefix
// bits n - (2^l - 1), oldest bit first.  Returns the context of the bit that
// follows `pos` plus that prefix.
__device__ __forceinline__ void node_context(const DecState &d, int n, uint32_t &h0, uint64_t &hist, int &c1) {
  int l = 31 - __clz(n + 1);
  uint32_t pb = (uint32_t)(n + 1 - (1 << l));
  int total = d.r + l;
  if (total < 8) {
    h0 = (1u << total) | (d.cur << l) | pb;
    hist = d.hist;
  } else {
    int m = 8 - d.r;                 // prefix bits that complete the current byte
    int rest = l - m;
    uint32_t done = ((d.cur << m) | (pb >> rest)) & 0xffu;
    h0 = (1u << rest) | (pb & ((1u << rest) - 1u));
    hist = (d.hist << 8) | done;
  }
  c1 = (int)(hist & 0xffu);
}

__device__ __forceinline__ uint32_t win_byte(const uint8_t *win, uint64_t win_base, uint64_t i, uint64_t plen) {
  return i < plen ? win[i - win_base] : 255u;
}

__device__ void decompress_one(const ChunkTask &t, uint8_t *slot, const Smem &s, const Layout &L,
                               const ModelInit *init, int spec, uint8_t *nodes) {
  const int tid = threadIdx.x;
  const int U = L.U;
  const uint64_t len = t.out_cap < t.cs ? t.out_cap : t.cs;  // bytes to decode
  const uint64_t nbits = 8ull * len;
  const uint8_t *pay = t.in;
  const uint64_t plen = t.in_len;
  uint8_t *out = t.out;

  // node arrays: nkey[8][255] u32, npr[256] u16, nfs[8][255] u8, ncxt[256] u8
  const int NN = 255;
  uint32_t *nkey = reinterpret_cast<uint32_t *>(nodes);
  uint16_t *npr = reinterpret_cast<uint16_t *>(nodes + kNodeKeyBytes);
  uint8_t *nfs = nodes + kNodeKeyBytes + kNodePrBytes;
  uint8_t *ncxt = nfs + kNodeFsBytes;
  uint8_t *win = s.stage;  // payload window
  __shared__ DecState sd;
  __shared__ uint64_t s_win_base;

  load_model(s, init, L);
  for (int i = tid; i < kWin; i += blockDim.x) win[i] = (uint64_t)i < plen ? pay[i] : 0;
  if (tid == 0) {
    s_win_base = 0;
    DecState d;
    d.x1 = 0;
    d.x2 = 0xffffffffu;
    d.x = 0;
    for (int i = 0; i < 4; i++) d.x = (d.x << 8) | ((uint64_t)i < plen ? pay[i] : 255u);  // cucm_decompress_v2.cu:967-972
    d.ioff = 4;
    d.pos = 0;
    d.hist = 0;
    d.cur = 0;
    d.r = 0;
    sd = d;
  }
  __syncthreads();

  for (uint64_t base = 0; base < nbits; base += U) {
    const int nunit = (int)(nbits - base < (uint64_t)U ? nbits - base : (uint64_t)U);
    int j = 0;
    while (j < nunit) {
      const int k = (nunit - j) < spec ? (nunit - j) : spec;
      const int nn = (1 << k) - 1;
      const DecState d = sd;
      // Keep the payload window ahead of the coder (at most 4 bytes per bit).
      // Every thread reads sd and s_win_base before the barrier; only then
      // may thread 0 move the window.
      const bool refill = d.ioff + 64 > s_win_base + kWin;
      __syncthreads();
      if (refill) {
        const uint64_t nb = d.ioff & ~(uint64_t)15;
        for (int i = tid; i < kWin; i += blockDim.x) win[i] = (nb + i < plen) ? pay[nb + i] : 0;
        if (tid == 0) s_win_base = nb;
      }
      // D1: keys and frozen states of every (node, order)
      for (int idx = tid; idx < nn * kOrders; idx += blockDim.x) {
        int n = idx >> 3, o = idx & 7;
        uint32_t h0;
        uint64_t hist;
        int c1;
        node_context(d, n, h0, hist, c1);
        BitKeys kk;
        bit_keys64(h0, hist, kk);
        nkey[o * NN + n] = kk.k[o];
        nfs[o * NN + n] = slot[table_offset(o) + kk.k[o]];
      }
      __syncthreads();
      // D2: mixer output of every node
      for (int n = tid; n < nn; n += blockDim.x) {
        uint32_t h0;
        uint64_t hist;
        int c1;
        node_context(d, n, h0, hist, c1);
        uint8_t st[kOrders];
#pragma unroll
        for (int o = 0; o < kOrders; o++) st[o] = nfs[o * NN + n];
        int smp[kOrders];
        int cx = stretch_and_cxt(s, st, c1, smp);
        npr[n] = (uint16_t)mix_pr(s.w, cx, smp, s.tab);
        ncxt[n] = (uint8_t)cx;
      }
      __syncthreads();
      // D3: decode k bits along the tree (decode, cucm_decompress_v2.cu:813-868)
      if (tid == 0) {
        DecState e = d;
        const uint64_t wbase = s_win_base;
        int n = 0;
        for (int i = 0; i < k; i++) {
          uint32_t pr = npr[n];
          uint32_t xmid = coder_mid(e.x1, e.x2, pr);
          int y = e.x <= xmid;
          if (y) e.x2 = xmid; else e.x1 = xmid + 1;
          while (((e.x1 ^ e.x2) & 0xff000000u) == 0) {
            e.x1 <<= 8;
            e.x2 = (e.x2 << 8) | 255u;
            e.x = (e.x << 8) | win_byte(win, wbase, e.ioff, plen);
            e.ioff++;
          }
          const int jj = j + i;
#pragma unroll
          for (int o = 0; o < kOrders; o++) {
            s.key[o * U + jj] = nkey[o * NN + n];
            s.fs[o * U + jj] = nfs[o * NN + n];
          }
          s.yb[jj] = (uint8_t)y;
          s.prm[jj] = (uint16_t)((pr << 1) | (uint32_t)y);
          s.cxt[jj] = ncxt[n];
          e.cur = (e.cur << 1) | (uint32_t)y;
          e.r++;
          if (e.r == 8) {
            out[e.pos >> 3] = (uint8_t)e.cur;
            e.hist = (e.hist << 8) | e.cur;
            e.cur = 0;
            e.r = 0;
          }
          e.pos++;
          n = 2 * n + 1 + y;
        }
        sd = e;
      }
      __syncthreads();
      j += k;
    }

    // Unit end: mixer deltas, then the StateMap chain, then write-back
    // (updateStateMap / updateMixer, cucm_decompress_v2.cu:870-896).
    for (int jj = tid; jj < nunit; jj += blockDim.x) {
      int smp[kOrders];
#pragma unroll
      for (int o = 0; o < kOrders; o++) smp[o] = s.tab->stretch[s.statep[o * 256 + s.fs[o * U + jj]] >> 20];
      mixer_train(s.w, s.cxt[jj], smp, s.yb[jj], s.prm[jj] >> 1);
    }
    __syncthreads();
    if (tid < kOrders) chain_order(s, L, tid, nunit);
    __syncthreads();
    write_back(s, L, slot);
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) decompress_kernel(const ChunkTask *tasks, uint32_t ntasks, uint8_t *slots,
                                                         const uint8_t *init_tables, const ModelInit *init,
                                                         uint32_t *queue, uint32_t *status, int unit, int spec) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  const Layout L = make_layout(unit, 0);
  const Smem s = carve(smem_raw, L);
  uint8_t *nodes = smem_raw + L.total;
  uint8_t *slot = slots + (size_t)blockIdx.x * kSlotTableBytes;
  copy_tables(&g_tables, s.tab);
  __shared__ uint32_t s_task;
  bool fresh = true;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_task = atomicAdd(queue, 1u);
    __syncthreads();
    const uint32_t ti = s_task;
    if (ti >= ntasks) break;
    const ChunkTask t = tasks[ti];
    if (t.unit != (uint32_t)unit || t.cs == 0) {
      if (threadIdx.x == 0) atomicOr(status, (uint32_t)kDevBadTask);
      continue;
    }
    if (!fresh) {
      reset_slot(slot, init_tables);
      __syncthreads();
    }
    fresh = false;
    decompress_one(t, slot, s, L, init, spec, nodes);
  }
}

#include "compress_fast.cuh"
#include "decompress_fast.cuh"
#include "fixed_model.cuh"

}  // namespace

size_t compress_smem_bytes(int unit) {
  return unit <= kFastMaxUnit ? make_fast_layout(unit).total : make_layout(unit, 0).total;
}
int compress_threads(int unit) { return unit <= kFastMaxUnit ? kFastThreads : 256; }
size_t decompress_smem_bytes(int unit, int spec_bits) {
  (void)spec_bits;
  return make_layout(unit, 0).total + kNodeBytes;
}

cudaError_t launch_fixed_encode(const FixedTask *d_tasks, const uint64_t *d_first, uint32_t ntasks, uint64_t total,
                                const uint8_t *image, const ModelInit *d_init, uint32_t *d_status, int sm_count,
                                cudaStream_t stream) {
  if (ntasks == 0) return cudaSuccess;
  if (total) {
    const uint64_t blocks = (total + kFixedThreads - 1) / kFixedThreads;
    const uint64_t cap = (uint64_t)(sm_count > 0 ? sm_count : 148) * 8;
    fixed_prob_kernel<<<(unsigned)std::min<uint64_t>(blocks, cap), kFixedThreads, 0, stream>>>(
        d_tasks, d_first, ntasks, total, image, d_init);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  // one warp of coders per CTA: the warps land on different SMs
  fixed_coder_kernel<<<(ntasks + 31) / 32, 32, 0, stream>>>(d_tasks, ntasks, d_status);
  return cudaGetLastError();
}

cudaError_t launch_fixed_decode(const FixedTask *d_tasks, uint32_t ntasks, const uint8_t *image,
                                const ModelInit *d_init, uint32_t *d_queue, int sm_count, cudaStream_t stream) {
  if (ntasks == 0) return cudaSuccess;
  // chunks spread over all SMs first: warps per CTA = chunks per SM, at
  // most kFixedDecWarps (each warp's rounds wait on its gathers, so warps
  // sharing an SM slow each other only through its load pipe)
  const uint32_t sms = (uint32_t)(sm_count > 0 ? sm_count : 148);
  const uint32_t warps = std::min<uint32_t>(kFixedDecWarps, (ntasks + sms - 1) / sms);
  const uint32_t want = (ntasks + warps - 1) / warps;
  fixed_decode_kernel<<<std::min(want, sms * 4), warps * 32, 0, stream>>>(d_tasks, ntasks, image, d_init, d_queue);
  return cudaGetLastError();
}

cudaError_t upload_tables() {
  Tables t;
  build_tables(t);
  return cudaMemcpyToSymbol(g_tables, &t, sizeof(Tables));
}

static cudaError_t set_smem(const void *fn, size_t bytes) {
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Pipelined compressor CTAs that fit on one SM: shared memory (1 KiB of it
// reserved per CTA by the hardware) and the registers of two CTAs
// (__launch_bounds__(kFastThreads, 2)).
static int fast_ctas_per_sm(int unit) {
  const size_t per = make_fast_layout(unit).total + 1024 + 64;
  const int by_smem = (int)((228u * 1024u) / per);
  const int by_regs = 2;
  const int n = by_smem < by_regs ? by_smem : by_regs;
  return n < 1 ? 1 : n;
}

cudaError_t launch_compress(const ChunkTask *d_tasks, uint32_t ntasks, uint8_t *slots, uint32_t nslots,
                            const uint8_t *init_tables, const ModelInit *d_init, uint32_t *d_queue,
                            uint32_t *d_status, const EngineConfig &cfg, cudaStream_t stream, int unit,
                            TailTask *tails, uint32_t *tail_count) {
  if (unit <= kFastMaxUnit && !cfg.generic) {
    const size_t smem = make_fast_layout(unit).total;
    const void *kern = unit <= 128 ? (const void *)compress_fast_kernel : (const void *)compress_fast_kernel_wide;
    cudaError_t e = set_smem(kern, smem);
    if (e != cudaSuccess) return e;
    if (unit <= 128)
      compress_fast_kernel<<<nslots, kFastThreads, smem, stream>>>(d_tasks, ntasks, slots, init_tables, d_init,
                                                                    d_queue, d_status, unit, tails, tail_count);
    else
      compress_fast_kernel_wide<<<nslots, kFastThreads, smem, stream>>>(d_tasks, ntasks, slots, init_tables, d_init,
                                                                         d_queue, d_status, unit, tails, tail_count);
    e = cudaGetLastError();
    if (e != cudaSuccess || !tails) return e;
    compress_tail_kernel<<<(ntasks + 127) / 128, 128, 0, stream>>>(tails, tail_count, d_status);
    return cudaGetLastError();
  }
  const size_t smem = make_layout(unit, 0).total;
  cudaError_t e = set_smem((const void *)compress_kernel, smem);
  if (e != cudaSuccess) return e;
  compress_kernel<<<nslots, 256, smem, stream>>>(d_tasks, ntasks, slots, init_tables, d_init, d_queue, d_status,
                                                 unit);
  return cudaGetLastError();
}

// Chunks (warp pairs) of the decoder that fit in one CTA's shared memory.
static int dec_max_pairs(int unit) {
  const DecLayout one = make_dec_layout(unit, 1);
  const size_t avail = kDecSmemLimit - (one.total - one.per_warp);
  int w = (int)(avail / one.per_warp);
  return w < 1 ? 1 : (w > kDecMaxPairs ? kDecMaxPairs : w);
}

static bool dec_fast(int unit, const EngineConfig &cfg) { return unit <= kDecMaxUnit && !cfg.generic; }

int engine_slots_per_sm(bool decode, int unit, const EngineConfig &cfg) {
  if (decode && dec_fast(unit, cfg))
    return cfg.dec_pairs > 0 ? std::min(cfg.dec_pairs, dec_max_pairs(unit)) : dec_max_pairs(unit);
  if (!decode && unit <= kFastMaxUnit && !cfg.generic) {
    const int fit = fast_ctas_per_sm(unit);
    return cfg.cmp_ctas > 0 && cfg.cmp_ctas < fit ? cfg.cmp_ctas : fit;
  }
  const size_t smem = decode ? decompress_smem_bytes(unit, cfg.spec_bits) : make_layout(unit, 0).total;
  return smem > 110 * 1024 ? 1 : (smem > 72 * 1024 ? 2 : 3);
}

cudaError_t launch_decompress(const ChunkTask *d_tasks, uint32_t ntasks, uint8_t *slots, uint32_t nslots,
                              const uint8_t *init_tables, const ModelInit *d_init, uint32_t *d_queue,
                              uint32_t *d_status, const EngineConfig &cfg, cudaStream_t stream, int unit) {
  if (dec_fast(unit, cfg)) {
    // One chunk per warp pair; spread the pairs over all SMs before stacking them.
    int sms = cfg.sm_count;
    if (sms <= 0) {
      int dev = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (sms <= 0) sms = 1;
    }
    int wpc = (int)((nslots + (uint32_t)sms - 1) / (uint32_t)sms);
    const int wmax = dec_max_pairs(unit);
    if (cfg.dec_pairs > 0) wpc = cfg.dec_pairs;
    if (wpc > wmax) wpc = wmax;
    if (wpc < 1) wpc = 1;
    // up to two chunks per CTA leave room for their order 0/1 tables in
    // shared memory
    const DecLayout Low = make_dec_layout(unit, wpc, true);
    const bool low = cfg.dec_tables == 0 && wpc <= 2 && Low.total <= kDecSmemLimit;
    const DecLayout L = low ? Low : make_dec_layout(unit, wpc);
    const void *kern = low ? (const void *)decompress_pair_kernel<true> : (const void *)decompress_pair_kernel<false>;
    cudaError_t e = set_smem(kern, L.total);
    if (e != cudaSuccess) return e;
    const uint32_t grid = (nslots + (uint32_t)wpc - 1) / (uint32_t)wpc;
    const uint32_t spin = cfg.spin_limit ? cfg.spin_limit : kDecSpinLimit;
    if (low)
      decompress_pair_kernel<true><<<grid, wpc * 64, L.total, stream>>>(d_tasks, ntasks, slots, nslots, init_tables,
                                                                        d_init, d_queue, d_status, unit, spin);
    else
      decompress_pair_kernel<false><<<grid, wpc * 64, L.total, stream>>>(d_tasks, ntasks, slots, nslots, init_tables,
                                                                         d_init, d_queue, d_status, unit, spin);
    return cudaGetLastError();
  }
  size_t smem = decompress_smem_bytes(unit, cfg.spec_bits);
  cudaError_t e = set_smem((const void *)decompress_kernel, smem);
  if (e != cudaSuccess) return e;
  int spec = cfg.spec_bits < 1 ? 1 : (cfg.spec_bits > 8 ? 8 : cfg.spec_bits);
  decompress_kernel<<<nslots, cfg.threads, smem, stream>>>(d_tasks, ntasks, slots, init_tables, d_init, d_queue,
                                                           d_status, unit, spec);
  return cudaGetLastError();
}

}  // namespace cucm
