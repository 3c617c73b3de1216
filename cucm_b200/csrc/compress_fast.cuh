// compress_fast.cuh -- pipelined chunk compressor for units of 32..256 bits.
//
// Included by engine_kernels.cu (shares its tables and coder helpers).
//
// The reference runs five launches per unit and a host round trip between
// them (cucm_compress_v2.cu:1067-1090).  Here one CTA of 14 warps codes a
// chunk with every stage of a unit overlapped with the others:
//
//   state warps (2..9, one per order): the bit-history side of the model.
//     A slot's state only depends on the bits coded in it, never on the
//     adaptive probabilities, so this pass runs a unit ahead of everything
//     else: it computes the keys, gathers the unit's slot states, resolves
//     repeats of a slot inside the unit (warp match + a small shared hash
//     table), emits for every (bit, order) the state the StateMap update will
//     see ("live") and the state the prediction sees ("frozen", the unit-start
//     value), and writes the unit's final states back to the slot tables
//     before gathering the next unit.
//   chain warp (0, lane = order): the only serial model chain left, the
//     StateMap probability updates in bit order (cucm_compress_v2.cu:592-601),
//     with the adaptation rate carried next to each probability so that a
//     step is a handful of ALU ops plus one shared-memory load.
//   mix warps (10..13, thread = bit): stretch, mixer context, dot product,
//     squash for the unit (cudamixUnit, cucm_compress_v2.cu:755-792) against
//     a snapshot of the probabilities taken when the previous chain finished,
//     then the mixer training deltas (cudaupdateMixer, :794-819).
//   coder warp (1): the binary arithmetic coder, one unit behind the mix.
//
// Tick t: state pass of unit t, chain and mix of unit t-1, coder of unit
// t-2.  After the last data unit the coder keeps coding the stale unit
// buffer up to the chunk end, exactly like cudaencodeUnit's missing input
// bound (cucm_compress_v2.cu:850-852).

constexpr int kFastWarps = 14;
constexpr int kFastThreads = kFastWarps * 32;
constexpr int kFastMaxUnit = 256;
constexpr int kWChain = 0, kWCoder = 1, kWState = 2, kWMix = 10;
constexpr int kMixThreads = 128;
constexpr int kSnapThreads = 32 + kMixThreads;

struct FastLayout {
  int U, NB, logNB, stage;
  size_t off_tab, off_rec, off_snap, off_w, off_htk, off_htl, off_hts, off_key, off_st, off_fr, off_yb, off_c1,
      off_prm, off_stage, total;
};

__host__ __device__ inline FastLayout make_fast_layout(int U) {
  FastLayout L;
  L.U = U;
  L.NB = next_pow2(2 * U);
  L.logNB = ilog2(L.NB);
  L.stage = next_pow2(4 * U + 1024);
  if (L.stage < kStageMin) L.stage = kStageMin;
  size_t o = 0;
  L.off_tab = o;   o += sizeof(Tables);
  L.off_rec = o;   o += sizeof(uint64_t) * kOrders * 256;
  L.off_snap = o;  o += sizeof(uint32_t) * kOrders * 256;
  L.off_w = o;     o += sizeof(int32_t) * kMixCtx * kOrders;
  L.off_htk = o;   o += sizeof(uint32_t) * kOrders * L.NB;
  L.off_htl = o;   o += (size_t)kOrders * L.NB;
  L.off_hts = o;   o += (size_t)kOrders * L.NB;
  L.off_key = o;   o += sizeof(uint32_t) * 2 * kOrders * U;
  L.off_st = o;    o += (size_t)2 * kOrders * U;
  L.off_fr = o;    o += (size_t)2 * U * kOrders;
  L.off_yb = o;    o += (size_t)4 * U;
  L.off_c1 = o;    o += (size_t)4 * (U / 8) + 16;
  o = (o + 15) & ~(size_t)15;
  L.off_prm = o;   o += sizeof(uint16_t) * 2 * U;
  o = (o + 15) & ~(size_t)15;
  L.off_stage = o; o += (size_t)L.stage;
  L.total = o;
  return L;
}

struct FastSmem {
  Tables *tab;
  uint64_t *rec;     // [8][256]  statep | dt[count] << 32
  uint32_t *snap;    // [8][256]  statep as of the last finished chain
  int32_t *w;        // [80*8]
  uint32_t *htk;     // [8][NB]   0 = empty, else key + 1
  uint8_t *htl;      // [8][NB]   latest state of the slot
  uint8_t *hts;      // [8][NB]   state of the slot at the unit start
  uint32_t *key;     // [2][8][U]
  uint8_t *st;       // [2][8][U] live state for the chain
  uint8_t *fr;       // [2][U][8] frozen state for the mix
  uint8_t *yb;       // [4][U]
  uint8_t *c1;       // [4][U/8]  previous byte of each byte of the unit
  uint16_t *prm;     // [2][U]
  uint8_t *stage;
};

__device__ inline FastSmem carve_fast(uint8_t *b, const FastLayout &L) {
  FastSmem s;
  s.tab = reinterpret_cast<Tables *>(b + L.off_tab);
  s.rec = reinterpret_cast<uint64_t *>(b + L.off_rec);
  s.snap = reinterpret_cast<uint32_t *>(b + L.off_snap);
  s.w = reinterpret_cast<int32_t *>(b + L.off_w);
  s.htk = reinterpret_cast<uint32_t *>(b + L.off_htk);
  s.htl = b + L.off_htl;
  s.hts = b + L.off_hts;
  s.key = reinterpret_cast<uint32_t *>(b + L.off_key);
  s.st = b + L.off_st;
  s.fr = b + L.off_fr;
  s.yb = b + L.off_yb;
  s.c1 = b + L.off_c1;
  s.prm = reinterpret_cast<uint16_t *>(b + L.off_prm);
  s.stage = b + L.off_stage;
  return s;
}

__device__ __forceinline__ void named_barrier(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// Input bytes of unit v for the key computation: window index k holds chunk
// byte v*U/8 - 7 + k (0 outside [0, len)); lane holds k = lane and lane+32.
__device__ __forceinline__ void load_unit_window(const uint8_t *in, uint64_t len, int U, int v, int lane,
                                                 uint32_t &w0, uint32_t &w1) {
  const int64_t b0 = (int64_t)v * (U / 8) - 7;
  const int64_t i0 = b0 + lane, i1 = b0 + lane + 32;
  const int nbytes = U / 8 + 7;
  w0 = (lane < nbytes && i0 >= 0 && (uint64_t)i0 < len) ? (uint32_t)__ldg(in + i0) : 0u;
  w1 = (lane + 32 < nbytes && i1 >= 0 && (uint64_t)i1 < len) ? (uint32_t)__ldg(in + i1) : 0u;
}

__device__ __forceinline__ uint32_t window_byte(uint32_t w0, uint32_t w1, int k) {
  uint32_t a = __shfl_sync(0xffffffffu, w0, k & 31);
  uint32_t b = __shfl_sync(0xffffffffu, w1, k & 31);
  return k < 32 ? a : b;
}

// State pass, step 1: keys of unit v for order o; gathers of the slot states
// into registers.  The order-0 warp also stores the unit's bits and the
// previous byte of each byte (needed by the chain and the mixer context).
__device__ __forceinline__ void fast_keys_and_gather(const FastSmem &s, const FastLayout &L, const uint8_t *slot,
                                                     int o, int lane, int v, int nvalid, uint32_t w0, uint32_t w1,
                                                     uint32_t gath[kFastMaxUnit / 32]) {
  const int U = L.U;
  uint32_t *key = s.key + ((v & 1) * kOrders + o) * U;
  uint8_t *yb = s.yb + (v & 3) * U;
  uint8_t *c1 = s.c1 + (v & 3) * (U / 8);
  const uint8_t *tab = slot + table_offset(o);
  CUCM_UNROLL
  for (int g = 0; g < kFastMaxUnit / 32; g++) {
    if (g < U / 32) {
      const int j = g * 32 + lane;
      const int q = j >> 3, r = j & 7;
      const uint32_t cur = window_byte(w0, w1, q + 7);
      const uint32_t h0 = (1u << r) | (cur >> (8 - r));
      uint32_t acc = (kFnvBasis ^ h0) * kFnvPrime;
      uint32_t prev1 = 0;
      for (int i = 1; i <= 7; i++) {
        const uint32_t hb = window_byte(w0, w1, q + 7 - i);
        if (i == 1) prev1 = hb;
        if (i <= o) acc = (acc ^ hb) * kFnvPrime;
      }
      const uint32_t k = o == 0 ? h0 : (o == 1 ? ((prev1 << 8) | h0) : (acc & (kSlots - 1)));
      if (j < nvalid) {
        key[j] = k;
        gath[g] = __ldcg(tab + k);
      }
      if (o == 0 && j < nvalid) {
        yb[j] = (uint8_t)((cur >> (7 - r)) & 1u);
        if (r == 0) c1[q] = (uint8_t)prev1;
      }
    }
  }
}

// State pass, step 2: resolve unit v of order o.  Groups of 32 bits in bit
// order; bits that share a slot inside a group are found with a warp match,
// across groups through a per-unit hash table (slot -> latest state, state
// at unit start).  The first touch of a slot in the unit starts from the
// gathered state.
__device__ __forceinline__ void fast_resolve(const FastSmem &s, const FastLayout &L, uint8_t *slot, int o, int lane,
                                             int v, int nvalid, const uint32_t gath[kFastMaxUnit / 32]) {
  const int U = L.U, NB = L.NB;
  uint32_t *htk = s.htk + o * NB;
  uint8_t *htl = s.htl + o * NB;
  uint8_t *hts = s.hts + o * NB;
  const uint32_t *key = s.key + ((v & 1) * kOrders + o) * U;
  const uint8_t *yb = s.yb + (v & 3) * U;
  uint8_t *st = s.st + ((v & 1) * kOrders + o) * U;
  uint8_t *fr = s.fr + (v & 1) * U * kOrders;
  const Tables *t = s.tab;
  for (int b = lane; b < NB; b += 32) htk[b] = 0;
  __syncwarp();
  CUCM_UNROLL
  for (int g = 0; g < kFastMaxUnit / 32; g++) {
    if (g < U / 32 && g * 32 < nvalid) {
      const int j = g * 32 + lane;
      const bool act = j < nvalid;
      const uint32_t k = act ? key[j] : (0x80000000u | (uint32_t)lane);
      const int y = act ? yb[j] : 0;
      const uint32_t peers = __match_any_sync(0xffffffffu, k);
      const int leader = __ffs(peers) - 1;
      const uint32_t lower = peers & ((1u << lane) - 1u);
      const int rank = __popc(lower);
      const int cnt = __popc(peers);
      int ss = 0, ls = 0, pos = 0;
      if (lane == leader && act) {
        // Leaders of distinct keys probe side by side, so an empty bucket is
        // claimed with a compare-and-swap; a lost race moves on.
        uint32_t b = bucket_of(k, L.logNB);
        for (;;) {
          uint32_t kk = htk[b];
          if (kk == 0) {
            kk = atomicCAS(&htk[b], 0u, k + 1);
            if (kk == 0) {
              ss = ls = (int)(gath[g] & 0xffu);
              hts[b] = (uint8_t)ss;
              break;
            }
          }
          if (kk == k + 1) {
            ss = hts[b];
            ls = htl[b];
            break;
          }
          b = (b + 1) & (uint32_t)(NB - 1);
        }
        pos = (int)b;
      }
      ss = __shfl_sync(0xffffffffu, ss, leader);
      ls = __shfl_sync(0xffffffffu, ls, leader);
      pos = __shfl_sync(0xffffffffu, pos, leader);
      // Repeats inside the group: the k-th peer sees the state left by the
      // (k-1)-th one.
      const int maxc = __reduce_max_sync(0xffffffffu, (unsigned)cnt);
      const int pred = rank ? 31 - __clz(lower) : lane;
      int cur = ls, ns = 0;
      for (int step = 0; step < maxc; step++) {
        if (rank == step) ns = t->nex[cur][y];
        const int vv = __shfl_sync(0xffffffffu, ns, pred);
        if (rank == step + 1) cur = vv;
      }
      if (act) {
        st[j] = (uint8_t)cur;
        fr[j * kOrders + o] = (uint8_t)ss;
        if (rank == cnt - 1) htl[pos] = (uint8_t)ns;
      }
      __syncwarp();
    }
  }
  // Final states of the unit go to the slot table before the next gather.
  uint8_t *tab = slot + table_offset(o);
  for (int b = lane; b < NB; b += 32) {
    const uint32_t kk = htk[b];
    if (kk) tab[kk - 1] = htl[b];
  }
  __syncwarp();
}

// Chain warp: StateMap probability updates of unit v in bit order, one lane
// per order.  rec[s] carries dt[count(s)] next to the probability so a step
// needs one shared load (issued a step early) and a few ALU ops; equal
// consecutive states forward the fresh value.
__device__ __forceinline__ void fast_chain(const FastSmem &s, const FastLayout &L, int o, int v, int n) {
  const int U = L.U;
  const uint8_t *sta = s.st + ((v & 1) * kOrders + o) * U;
  const uint8_t *yb = s.yb + (v & 3) * U;
  uint64_t *rec = s.rec + o * 256;
  const uint16_t *dt = s.tab->dt;
  int st = sta[0];
  int st1 = n > 1 ? sta[1] : 0;
  uint64_t r = rec[st];
  for (int j = 0; j < n; j++) {
    const uint64_t r1 = rec[st1];
    const int st2 = (j + 2 < n) ? sta[j + 2] : 0;
    const uint32_t y = yb[j];
    const uint32_t val = (uint32_t)r, d = (uint32_t)(r >> 32);
    const uint32_t cnt = val & 1023u;
    const int32_t err = (int32_t)((y << 22) - (val >> 10));
    const uint32_t v2 = val + (((uint32_t)(err >> 3) * d) & 0xfffffc00u) + (cnt < 1023u ? 1u : 0u);
    const uint32_t d2 = dt[cnt < 1023u ? cnt + 1 : 1023u];
    const uint64_t nr = (uint64_t)v2 | ((uint64_t)d2 << 32);
    rec[st] = nr;
    r = (st1 == st) ? nr : r1;
    st = st1;
    st1 = st2;
  }
}

// Mix warps: predictions, mixer output and training of unit v; thread t
// handles bits t and t + 128.
__device__ __forceinline__ void fast_mix(const FastSmem &s, const FastLayout &L, int t, int v, int nvalid) {
  const int U = L.U;
  const uint8_t *fr = s.fr + (v & 1) * U * kOrders;
  const uint8_t *yb = s.yb + (v & 3) * U;
  const uint8_t *c1 = s.c1 + (v & 3) * (U / 8);
  uint16_t *prm = s.prm + (v & 1) * U;
  const uint16_t *prm_old = s.prm + ((v + 1) & 1) * U;
  const Tables *tb = s.tab;
  int cxs[2] = {0, 0}, errs[2] = {0, 0};
  int smps[2][kOrders];
  bool has[2] = {false, false};
  CUCM_UNROLL
  for (int h = 0; h < 2; h++) {
    const int j = t + h * kMixThreads;
    if (j < U) {
      if (j < nvalid) {
        const uint64_t f8 = *reinterpret_cast<const uint64_t *>(fr + j * kOrders);
        int olen = 0;
        CUCM_UNROLL
        for (int o = 0; o < kOrders; o++) {
          const uint32_t stt = (uint32_t)(f8 >> (8 * o)) & 0xffu;
          const int sm = tb->stretch[s.snap[o * 256 + stt] >> 20];
          smps[h][o] = sm;
          olen += (sm != 1);
        }
        const int cx = olen + (c1[j >> 3] >> 5) * 10;
        const int pr = mix_pr(s.w, cx, smps[h], tb);
        const int y = yb[j];
        prm[j] = (uint16_t)((pr << 1) | y);
        cxs[h] = cx;
        errs[h] = ((y << 12) - pr) * 7;
        has[h] = true;
      } else {
        prm[j] = prm_old[j];  // stale entry, re-coded as the reference does
      }
    }
  }
  named_barrier(2, kMixThreads);  // every weight read before any update
  CUCM_UNROLL
  for (int h = 0; h < 2; h++) {
    if (has[h]) {
      CUCM_UNROLL
      for (int o = 0; o < kOrders; o++) {
        const int d = (int)(((long long)errs[h] * smps[h][o]) >> 16);
        atomicAdd(&s.w[cxs[h] * kOrders + o], d);
      }
    }
  }
}

__device__ void compress_fast_one(const ChunkTask &t, uint8_t *slot, const FastSmem &s, const FastLayout &L,
                                  const ModelInit *init, uint32_t *status) {
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int U = L.U;
  const uint64_t len = t.in_len < t.cs ? t.in_len : t.cs;
  const uint64_t total_bits = 8ull * t.cs;
  const uint64_t data_bits = 8ull * len;
  const int nU = (int)((data_bits + U - 1) / U);
  auto nvalid_of = [&](int v) -> int {
    const uint64_t b = (uint64_t)v * U;
    return b >= data_bits ? 0 : (int)(data_bits - b < (uint64_t)U ? data_bits - b : (uint64_t)U);
  };
  auto ncode_of = [&](int v) -> int {
    const uint64_t b = (uint64_t)v * U;
    return b >= total_bits ? 0 : (int)(total_bits - b < (uint64_t)U ? total_bits - b : (uint64_t)U);
  };

  for (int i = tid; i < kOrders * 256; i += blockDim.x) {
    const uint32_t v = init->statep[i >> 8][i & 255];
    s.rec[i] = (uint64_t)v | ((uint64_t)s.tab->dt[v & 1023u] << 32);
  }
  for (int i = tid; i < kMixCtx * kOrders; i += blockDim.x) s.w[i] = init->w[i];
  for (int i = tid; i < 2 * U; i += blockDim.x) s.prm[i] = 0;  // cucm_compress_v2.cu:1039-1040

  Coder c{0u, 0xffffffffu, 0, 0};
  uint32_t gath[kFastMaxUnit / 32];
  uint32_t w0 = 0, w1 = 0;
  const bool is_state = warp >= kWState && warp < kWMix;
  const int so = warp - kWState;
  if (is_state) {
    uint32_t a0, a1;
    load_unit_window(t.in, len, U, 0, lane, a0, a1);
    __syncthreads();
    fast_keys_and_gather(s, L, slot, so, lane, 0, nvalid_of(0), a0, a1, gath);
    if (nU > 1) load_unit_window(t.in, len, U, 1, lane, w0, w1);
  } else {
    __syncthreads();
  }
  __syncthreads();

  for (int tau = 0; tau < nU + 2; tau++) {
    const int um = tau - 1;
    const bool snap_role = warp == kWChain || warp >= kWMix;
    if (snap_role) {
      if (um >= 0 && um < nU) {
        const int k = warp == kWChain ? lane : 32 + (tid - kWMix * 32);
        for (int i = k; i < kOrders * 256; i += kSnapThreads) s.snap[i] = (uint32_t)s.rec[i];
      }
      named_barrier(1, kSnapThreads);
    }
    if (warp == kWChain) {
      if (um >= 0 && um < nU && lane < kOrders) fast_chain(s, L, lane, um, nvalid_of(um));
    } else if (warp == kWCoder) {
      const int uc = tau - 2;
      if (uc >= 0 && uc < nU) {
        coder_run_p(c, s.prm + (uc & 1) * U, s.stage, L.stage, ncode_of(uc));
        coder_flush_p(c, s.stage, L.stage, t.out, t.out_cap);
      }
    } else if (is_state) {
      if (tau < nU) {
        fast_resolve(s, L, slot, so, lane, tau, nvalid_of(tau), gath);
        if (tau + 1 < nU) {
          fast_keys_and_gather(s, L, slot, so, lane, tau + 1, nvalid_of(tau + 1), w0, w1, gath);
          if (tau + 2 < nU) load_unit_window(t.in, len, U, tau + 2, lane, w0, w1);
        }
      }
    } else {
      if (um >= 0 && um < nU) fast_mix(s, L, tid - kWMix * 32, um, nvalid_of(um));
    }
    __syncthreads();
  }

  if (warp == kWCoder) {
    const uint16_t *last = s.prm + ((nU - 1) & 1) * U;
    for (int v = nU; ; v++) {
      const int n = ncode_of(v);
      if (n <= 0) break;
      coder_run_p(c, last, s.stage, L.stage, n);
      coder_flush_p(c, s.stage, L.stage, t.out, t.out_cap);
    }
    coder_finish_p(c, s.stage, L.stage, t.out, t.out_cap, t.result);
    if (lane == 0 && c.head > t.out_cap) atomicOr(status, (uint32_t)kDevOverflow);
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kFastThreads, 2)
    compress_fast_kernel(const ChunkTask *tasks, uint32_t ntasks, uint8_t *slots, const uint8_t *init_tables,
                         const ModelInit *init, uint32_t *queue, uint32_t *status, int unit) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  const FastLayout L = make_fast_layout(unit);
  const FastSmem s = carve_fast(smem_raw, L);
  uint8_t *slot = slots + (size_t)blockIdx.x * kSlotTableBytes;
  copy_tables(s.tab);
  __shared__ uint32_t s_task;
  bool fresh = true;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_task = atomicAdd(queue, 1u);
    __syncthreads();
    const uint32_t ti = s_task;
    if (ti >= ntasks) break;
    const ChunkTask t = tasks[ti];
    if (t.unit != (uint32_t)unit || t.cs == 0 || t.in_len == 0) {
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
    compress_fast_one(t, slot, s, L, init, status);
  }
}
