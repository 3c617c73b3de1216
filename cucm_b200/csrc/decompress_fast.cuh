// decompress_fast.cuh -- chunk decoder, two warps per chunk, units of 32..256 bits.
//
// Included by engine_kernels.cu (shares its tables and helpers).
//
// The reference decodes a unit in speculation steps of L+1 bits, each step
// three launches and a host round trip (cucm_decompress_v2.cu:977-1032).
// Here a pair of warps owns a chunk and decodes it a nibble ("round") at a
// time.
//
// The decoding warp:
//   * gives the 15 nodes of the nibble's speculation tree (every prefix of
//     0..3 bits) their 8 context keys and frozen slot states -- one lane per
//     node, its 6 hashed orders' gathers in flight together (orders 0 and 1
//     come from shared memory when the CTA has room for them), so a round
//     costs one memory round trip;
//   * mixes and squashes each node's prediction against the frozen model
//     (probabilities kept stretched) and decodes the 4 bits uniformly (every
//     lane runs the same coder arithmetic; the split point of a node comes
//     from its lane by shuffle);
//   * has the 4 lanes on the decoded path record keys, states and mixer
//     inputs of their bit in a per-unit ring, and publishes the round.
// The updating warp follows one round behind (lane = order), polling for
// published rounds: the bit-history walk through a per-unit overlay (slot ->
// live state, 4-key buckets), the StateMap probability chain and the mixer
// deltas, all in bit order.  Nothing the decoding warp reads changes before
// the unit ends, so the two only meet there: the overlay's states go to the
// slot tables, the live probabilities become the frozen ones and the summed
// mixer deltas join the weights (updateStateMap / updateMixer,
// cucm_decompress_v2.cu:870-896).  Rounds never straddle a unit or byte
// boundary: units are multiples of 32 bits.
//
// Several warp pairs of a CTA decode independent chunks and share the
// read-only tables.

constexpr int kDecMaxUnit = 256;
constexpr int kDecMaxPairs = 8;          // chunks per CTA
constexpr int kDecWin = 2048;            // payload window per chunk (bytes)
constexpr int kDecNodes = 15;            // nodes of a 4-bit speculation tree
constexpr size_t kDecSmemLimit = 227 * 1024;  // dynamic shared memory of one CTA
constexpr uint32_t kDecSpinLimit = 1u << 27;  // default bound on the updater's polls for a round (seconds)

struct DecLayout {
  int U, NS, logNS, warps, rounds;
  bool low;  // order 0/1 tables held in shared memory
  size_t off_spf, off_spl, off_w, off_dw, off_ovk, off_ovs, off_ovl, off_ovn, off_prog, off_rk, off_rs, off_rsmp,
      off_rpc, off_win, off_outb, off_t01, per_warp, off_tab, total;
};

// Shared memory of `warps` chunks (warp pairs) and the shared tables.
// With `low`, each chunk also holds its order 0 and 1 tables (the first
// kHashedOff bytes of its slot, 64.25 KiB) in shared memory.
__host__ __device__ inline DecLayout make_dec_layout(int U, int warps, bool low = false) {
  DecLayout L;
  L.U = U;
  L.low = low;
  L.rounds = U / 4;
  L.NS = next_pow2(2 * U);  // overlay slots per order (load <= 1/2)
  L.logNS = ilog2(L.NS);
  L.warps = warps;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    size_t at = o;
    o = (o + bytes + 15) & ~(size_t)15;
    return at;
  };
  L.off_spf = take(sizeof(int16_t) * 256 * kOrders);           // frozen probability, stretched [state][order]
  L.off_spl = take(sizeof(uint32_t) * 256 * kOrders);          // live statep [state][order]
  L.off_w = take(sizeof(int32_t) * kMixCtx * kOrders);         // frozen weights
  L.off_dw = take(sizeof(int32_t) * kMixCtx * kOrders);        // summed deltas of the unit
  L.off_ovk = take(sizeof(uint32_t) * kOrders * L.NS);         // overlay keys + 1 (0 = empty), 4-key buckets
  L.off_ovs = take((size_t)kOrders * L.NS);                    // overlay live states
  L.off_ovl = take(sizeof(uint16_t) * U * kOrders);            // overlay entries in use [entry][order]
  L.off_ovn = take(sizeof(int) * kOrders);
  L.off_prog = take(sizeof(uint32_t) * 4);                     // rounds published; task index
  L.off_rk = take(sizeof(uint32_t) * L.rounds * 4 * kOrders);  // records [round][bit][order]
  L.off_rs = take((size_t)L.rounds * 4 * kOrders);
  L.off_rsmp = take(sizeof(int16_t) * L.rounds * 4 * kOrders);
  L.off_rpc = take(sizeof(uint32_t) * L.rounds * 4);           // pr | cxt << 16 | y << 24
  L.off_win = take((size_t)kDecWin);
  L.off_outb = take((size_t)kDecMaxUnit / 8);
  L.off_t01 = low ? take((size_t)kHashedOff) : 0;
  L.per_warp = o;
  L.off_tab = (size_t)warps * L.per_warp;
  L.total = L.off_tab + ((sizeof(Tables) + 15) & ~(size_t)15);
  return L;
}

struct DecSmem {
  int16_t *spf;
  uint32_t *spl;
  int32_t *w, *dw;
  uint32_t *ovk;
  uint8_t *ovs;
  uint16_t *ovl;
  int *ovn;
  volatile uint32_t *prog;
  uint32_t *rk;
  uint8_t *rs;
  int16_t *rsmp;
  uint32_t *rpc;
  uint8_t *win, *outb;
  uint8_t *t01;  // order 0/1 tables, or null
};

__device__ inline DecSmem carve_dec(uint8_t *base, const DecLayout &L, int warp) {
  uint8_t *b = base + (size_t)warp * L.per_warp;
  DecSmem s;
  s.spf = reinterpret_cast<int16_t *>(b + L.off_spf);
  s.spl = reinterpret_cast<uint32_t *>(b + L.off_spl);
  s.w = reinterpret_cast<int32_t *>(b + L.off_w);
  s.dw = reinterpret_cast<int32_t *>(b + L.off_dw);
  s.ovk = reinterpret_cast<uint32_t *>(b + L.off_ovk);
  s.ovs = b + L.off_ovs;
  s.ovl = reinterpret_cast<uint16_t *>(b + L.off_ovl);
  s.ovn = reinterpret_cast<int *>(b + L.off_ovn);
  s.prog = reinterpret_cast<volatile uint32_t *>(b + L.off_prog);
  s.rk = reinterpret_cast<uint32_t *>(b + L.off_rk);
  s.rs = b + L.off_rs;
  s.rsmp = reinterpret_cast<int16_t *>(b + L.off_rsmp);
  s.rpc = reinterpret_cast<uint32_t *>(b + L.off_rpc);
  s.win = b + L.off_win;
  s.outb = b + L.off_outb;
  s.t01 = L.low ? b + L.off_t01 : nullptr;
  return s;
}

// One slot state from the tables in HBM (L2-cached load).  The memory
// clobber keeps the load where it is written: a round's gathers go out
// before the previous round's record is stored to shared memory.
__device__ __forceinline__ uint32_t ld_slot_state(const uint8_t *p) {
  uint32_t v;
  asm volatile("ld.global.cg.u8 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Warp-wide refill of the payload window so that it starts at or just below
// payload byte `at`, on a 16-byte boundary of the payload's address (so the
// window base may lie up to 15 bytes before the payload).  Only 16-byte
// blocks that hold payload bytes are read.  Returns the payload offset of
// window byte 0.
__device__ inline long long dec_refill(uint8_t *win, const uint8_t *pay, uint64_t plen, uint64_t at, int lane) {
  const uint8_t *a = reinterpret_cast<const uint8_t *>((reinterpret_cast<uintptr_t>(pay) + at) & ~(uintptr_t)15);
  const uint8_t *end = pay + plen;
  for (int j = lane; j < kDecWin / 16; j += 32) {
    const uint8_t *blk = a + 16 * j;
    if (blk < end) *reinterpret_cast<uint4 *>(win + 16 * j) = *reinterpret_cast<const uint4 *>(blk);
  }
  __syncwarp();
  return (long long)(a - pay);
}

// Overlay buckets hold 4 keys (+ 1, 0 = empty), filled in order and never
// emptied within a unit; a key whose bucket is full lives in the next bucket
// with room.  Place of `want` in bucket q, or -1:
__device__ __forceinline__ int bucket_place(const uint4 &q, uint32_t want) {
  return q.x == want ? 0 : q.y == want ? 1 : q.z == want ? 2 : q.w == want ? 3 : -1;
}
__device__ __forceinline__ int bucket_used(const uint4 &q) {
  return (q.x != 0u) + (q.y != 0u) + (q.z != 0u) + (q.w != 0u);
}

// Model update of one round's 4 bits for order `o` (one lane per order), in
// bit order: the live state of each slot (overlay, else the frozen state the
// prediction saw), its next state, the StateMap probability of the live state
// (cucm_decompress_v2.cu:870-883) and the mixer deltas (:885-896).
//
// All shared-memory reads of the four bits are issued before any write:
// what an earlier bit of the round changes for a later one -- the same
// slot's state, the same state's probability, an overlay entry it claims --
// is carried forward in registers, and the writes follow in bit order, so a
// later write to the same place wins as it would one bit at a time.
// `nov` is this lane's count of overlay entries in use (its order's list).
__device__ __forceinline__ void dec_update_round(const DecSmem &s, const Tables *tab, const DecLayout &L, int o,
                                                 int rd, int &nov) {
  uint32_t *ovk = s.ovk + o * L.NS;
  uint8_t *ovs = s.ovs + o * L.NS;
  const uint32_t bmask = (uint32_t)(L.NS / 4 - 1);
  uint32_t k[4], b[4], e[4] = {0, 0, 0, 0};
  int fz[4], sm[4], y[4];
  int cx[4], dl[4];
CUCM_UNROLL
  for (int i = 0; i < 4; i++) {
    const int r = (rd * 4 + i) * kOrders + o;
    k[i] = s.rk[r];
    fz[i] = s.rs[r];
    sm[i] = s.rsmp[r];
    const uint32_t pc = s.rpc[rd * 4 + i];
    y[i] = (int)(pc >> 24) & 1;
    const int pr = (int)(pc & 0xffffu);
    cx[i] = (int)(pc >> 16) & 0xff;
    dl[i] = (int)(((long long)(((y[i] << 12) - pr) * 7) * sm[i]) >> 16);
    b[i] = bucket_of(k[i], L.logNS - 2);
  }
  // mixer deltas (Mixer::update, cucm_compress_v2.cu:663-678): this lane
  // alone owns column o of the delta rows; deltas of the round's bits that
  // share a row are summed first (integer adds commute), then every distinct
  // row is read and written once
  bool merged[4] = {false, false, false, false};
CUCM_UNROLL
  for (int i = 1; i < 4; i++)
CUCM_UNROLL
    for (int j = 0; j < i; j++)
      if (!merged[i] && !merged[j] && cx[j] == cx[i]) {
        dl[j] += dl[i];
        merged[i] = true;
      }
  int dv[4];
CUCM_UNROLL
  for (int i = 0; i < 4; i++) dv[i] = s.dw[cx[i] * kOrders + o];
  // the four bits' buckets: keys and states
  const uint4 *ovk4 = reinterpret_cast<const uint4 *>(ovk);
  const uint32_t *ovs4 = reinterpret_cast<const uint32_t *>(ovs);
  uint4 q[4];
  uint32_t qs[4];
CUCM_UNROLL
  for (int i = 0; i < 4; i++) {
    q[i] = ovk4[b[i]];
    qs[i] = ovs4[b[i]];
  }
  // slots and live states, in bit order; e = slot (bucket * 4 + place)
  int live[4], ns[4];
  bool fresh[4];
CUCM_UNROLL
  for (int i = 0; i < 4; i++) {
    bool same = false;
    int lv = 0;
CUCM_UNROLL
    for (int j = 0; j < i; j++)
      if (k[j] == k[i]) {
        same = true;
        lv = ns[j];
        e[i] = e[j];
      }
    fresh[i] = false;
    if (!same) {
      const uint32_t want = k[i] + 1;
      const int hit = bucket_place(q[i], want);
      if (hit >= 0) {
        e[i] = b[i] * 4 + (uint32_t)hit;
        lv = (int)(qs[i] >> (8 * hit)) & 0xff;
      } else {
        // places this round has already claimed in the bucket
        int used = bucket_used(q[i]);
CUCM_UNROLL
        for (int j = 0; j < i; j++) used += (fresh[j] && (e[j] >> 2) == b[i]);
        if (used < 4) {
          e[i] = b[i] * 4 + (uint32_t)used;
          lv = fz[i];
          fresh[i] = true;
        } else {
          // full bucket: the key is in a later one, or goes to the first
          // with room
          uint32_t bi = b[i];
          for (uint32_t it = 0; it <= bmask; it++) {
            bi = (bi + 1) & bmask;
            const uint4 qq = ovk4[bi];
            const int h = bucket_place(qq, want);
            if (h >= 0) {
              e[i] = bi * 4 + (uint32_t)h;
              lv = ovs[e[i]];
              break;
            }
            int u = bucket_used(qq);
CUCM_UNROLL
            for (int j = 0; j < i; j++) u += (fresh[j] && (e[j] >> 2) == bi);
            if (u < 4) {
              e[i] = bi * 4 + (uint32_t)u;
              lv = fz[i];
              fresh[i] = true;
              break;
            }
          }
        }
      }
    }
    live[i] = lv;
    ns[i] = tab->nex[lv][y[i]];
  }
  // StateMap probabilities of the live states: a state met m times earlier
  // in the round has count min(count + m, 1023), so every dt is read up front
  uint32_t v0[4], dtv[4];
  int m[4];
CUCM_UNROLL
  for (int i = 0; i < 4; i++) {
    v0[i] = s.spl[live[i] * kOrders + o];
    m[i] = 0;
CUCM_UNROLL
    for (int j = 0; j < i; j++) m[i] += (live[j] == live[i]);
    const uint32_t c = (v0[i] & 1023u) + (uint32_t)m[i];
    dtv[i] = tab->dt[c > 1023u ? 1023u : c];
  }
  uint32_t nv[4];
CUCM_UNROLL
  for (int i = 0; i < 4; i++) {
    uint32_t v = v0[i];
CUCM_UNROLL
    for (int j = 0; j < i; j++)
      if (live[j] == live[i]) v = nv[j];
    nv[i] = statep_next(v, y[i], dtv[i]);
  }
  // writes, in bit order
CUCM_UNROLL
  for (int i = 0; i < 4; i++)
    if (!merged[i]) s.dw[cx[i] * kOrders + o] = dv[i] + dl[i];
CUCM_UNROLL
  for (int i = 0; i < 4; i++) {
    if (fresh[i]) {
      ovk[e[i]] = k[i] + 1;
      s.ovl[nov * kOrders + o] = (uint16_t)e[i];
      nov++;
    }
    ovs[e[i]] = (uint8_t)ns[i];
    s.spl[live[i] * kOrders + o] = nv[i];
  }
}

// Unit end, both warps of the pair (t = 0..63): overlay -> slot tables (and
// cleared), live probabilities become frozen (stretched for the mixer),
// deltas join the weights, the unit's bytes go out.  Called between two pair
// barriers.
__device__ inline void dec_unit_end(const DecSmem &s, const DecLayout &L, const Tables *tab, uint8_t *slot,
                                    uint8_t *out, int nbytes, int t) {
CUCM_UNROLL
  for (int o = 0; o < kOrders; o++) {
    const int n = s.ovn[o];
    uint8_t *tb = (o < 2 && s.t01 ? s.t01 : slot) + table_offset(o);
    for (int e = t; e < n; e += 64) {
      const int b = s.ovl[e * kOrders + o];
      const uint32_t kk = s.ovk[o * L.NS + b];
      tb[kk - 1] = s.ovs[o * L.NS + b];
      s.ovk[o * L.NS + b] = 0;
    }
  }
  const uint4 *src = reinterpret_cast<const uint4 *>(s.spl);
  uint2 *dst = reinterpret_cast<uint2 *>(s.spf);
  const int16_t *str = tab->stretch;
#pragma unroll 4
  for (int i = t; i < 256 * kOrders / 4; i += 64) {
    const uint4 q = src[i];
    const uint32_t a = (uint16_t)str[q.x >> 20], b = (uint16_t)str[q.y >> 20];
    const uint32_t c = (uint16_t)str[q.z >> 20], d = (uint16_t)str[q.w >> 20];
    dst[i] = make_uint2(a | (b << 16), c | (d << 16));
  }
  int4 *w4 = reinterpret_cast<int4 *>(s.w);
  int4 *d4 = reinterpret_cast<int4 *>(s.dw);
  for (int i = t; i < kMixCtx * kOrders / 4; i += 64) {
    int4 a = w4[i];
    const int4 d = d4[i];
    a.x += d.x;
    a.y += d.y;
    a.z += d.z;
    a.w += d.w;
    w4[i] = a;
    d4[i] = make_int4(0, 0, 0, 0);
  }
  if (t < nbytes) out[t] = s.outb[t];
}

// The pair's barrier: named barrier 1 + pair index, 64 threads.
__device__ __forceinline__ void pair_sync(int pair) {
  asm volatile("bar.sync %0, 64;" ::"r"(1 + pair) : "memory");
}

// One chunk.  role 0 decodes, role 1 updates the model; lane = threadIdx & 31.
template <bool kLow>
__device__ void decompress_pair_one(const ChunkTask &t, uint8_t *slot, const DecSmem &s, const Tables *tab,
                                    const DecLayout &L, const ModelInit *init, int role, int pair,
                                    uint32_t *status, uint32_t spin_limit) {
  const int lane = threadIdx.x & 31;
  const int t64 = lane + 32 * role;
  const int U = L.U;
  const uint64_t len = t.out_cap < t.cs ? t.out_cap : t.cs;  // bytes to decode
  const uint64_t nbits = 8ull * len;
  const uint8_t *pay = t.in;
  const uint64_t plen = t.in_len;

  for (int i = t64; i < 256 * kOrders; i += 64) {
    const uint32_t v = init->statep[i & 7][i >> 3];
    s.spf[i] = tab->stretch[v >> 20];
    s.spl[i] = v;
  }
  for (int i = t64; i < kMixCtx * kOrders; i += 64) {
    s.w[i] = init->w[i];
    s.dw[i] = 0;
  }
  for (int i = t64; i < kOrders * L.NS; i += 64) s.ovk[i] = 0;
  if (kLow) {
    // the chunk's order 0/1 tables move to shared memory for its lifetime
    const uint4 *src = reinterpret_cast<const uint4 *>(slot);
    uint4 *dst = reinterpret_cast<uint4 *>(s.t01);
    for (int i = t64; i < (int)(kHashedOff / 16); i += 64) dst[i] = src[i];
  }
  if (t64 < kOrders) s.ovn[t64] = 0;
  if (t64 == 0) s.prog[0] = 0;
  pair_sync(pair);

  if (role == 1) {
    // the updating warp: rounds in order, as the decoding warp publishes them
    uint32_t done = 0;
    bool ok = true;
    for (uint64_t base = 0; base < nbits; base += (uint64_t)U) {
      const int nunit = (int)(nbits - base < (uint64_t)U ? nbits - base : (uint64_t)U);
      int nov = 0;
      for (int rd = 0; rd < (nunit >> 2); rd++) {
        uint32_t spins = 0;
        while (ok && s.prog[0] <= done) {
          // a plain poll: a sleep here wakes late and the updating warp
          // falls rounds behind by the unit's end
          if (++spins >= spin_limit) ok = false;
        }
        __threadfence_block();
        if (!ok) break;
        if (lane < kOrders) dec_update_round(s, tab, L, lane, rd, nov);
        done++;
      }
      if (lane < kOrders) s.ovn[lane] = nov;
      if (!ok && lane == 0) atomicOr(status, (uint32_t)kDevTimeout);
      pair_sync(pair);
      dec_unit_end(s, L, tab, slot, t.out + (base >> 3), nunit >> 3, t64);
      pair_sync(pair);
    }
    return;
  }

  long long wbase = dec_refill(s.win, pay, plen, 0, lane);

  // coder state, identical in every lane (cucm_decompress_v2.cu:967-972)
  uint32_t x1 = 0, x2 = 0xffffffffu, x = 0;
  uint64_t ioff = 0;
  for (int i = 0; i < 4; i++, ioff++) x = (x << 8) | (ioff < plen ? (uint32_t)s.win[(long long)ioff - wbase] : 255u);

  // node of this lane (lanes 15..31 mirror lanes 0..14 so every gather
  // instruction stays uniform; only lanes < 15 record)
  const int node = lane % kDecNodes;
  const int depth = 31 - __clz(node + 1);
  const uint32_t pbits = (uint32_t)(node + 1 - (1 << depth));
  const bool recorder = lane < kDecNodes;

  uint64_t hist = 0;  // completed bytes, most recent in the low byte
  uint32_t cur = 0;   // bits of the current byte
  int r = 0;          // 0 or 4
  uint32_t published = 0;

  // A round's keys and frozen slot states.  After a round is decoded the
  // next round's gathers go out at once (within a unit: the unit end writes
  // the slot tables), and the decoded round is recorded and published while
  // they are in flight.
  BitKeys kk;
  uint32_t st[kOrders];
  auto gather = [&](BitKeys &k, uint32_t *sv, uint32_t cur_, int r_, uint64_t hist_) {
    const uint32_t h0 = (1u << (r_ + depth)) | (cur_ << depth) | pbits;
    bit_keys64(h0, hist_, k);
    if (kLow) {
      sv[0] = s.t01[k.k[0]];
      sv[1] = s.t01[kOrder1Off + k.k[1]];
    }
CUCM_UNROLL
    for (int o = kLow ? 2 : 0; o < kOrders; o++) sv[o] = ld_slot_state(slot + table_offset(o) + k.k[o]);
  };

  for (uint64_t base = 0; base < nbits; base += (uint64_t)U) {
    const int nunit = (int)(nbits - base < (uint64_t)U ? nbits - base : (uint64_t)U);
    const int nr = nunit >> 2;
    int obyte = 0;
    gather(kk, st, cur, r, hist);
    for (int rd = 0; rd < nr; rd++) {
      if ((long long)ioff + 16 > wbase + kDecWin) wbase = dec_refill(s.win, pay, plen, ioff, lane);
      // stretch, mixer context, mixer output (cucm_decompress_v2.cu:774-809)
      const int c1 = (int)(hist & 0xffu);
      int smp[kOrders];
      int olen = 0;
CUCM_UNROLL
      for (int o = 0; o < kOrders; o++) {
        smp[o] = s.spf[st[o] * kOrders + o];
        olen += (smp[o] != 1);
      }
      const int cxt = olen + (c1 >> 5) * 10;
      const int pr_node = mix_pr(s.w, cxt, smp, tab);
      // decode 4 bits along the tree (cucm_decompress_v2.cu:813-868); both
      // children's split factors are fetched while a bit is decided, so the
      // shuffle is off the bit-to-bit chain
      const uint32_t f_node = (uint32_t)pr_node << 20;
      int n = 0;
      uint32_t nib = 0;
      uint32_t f = __shfl_sync(0xffffffffu, f_node, 0);
CUCM_UNROLL
      for (int i = 0; i < 4; i++) {
        uint32_t fa = 0, fb = 0;
        if (i < 3) {
          fa = __shfl_sync(0xffffffffu, f_node, 2 * n + 1);
          fb = __shfl_sync(0xffffffffu, f_node, 2 * n + 2);
        }
        const uint32_t xm = x1 + __umulhi(x2 - x1, f);
        const int y = x <= xm;
        if (y) x2 = xm; else x1 = xm + 1;
        while ((x1 ^ x2) < 0x1000000u) {
          x1 <<= 8;
          x2 = (x2 << 8) | 255u;
          x = (x << 8) | (ioff < plen ? (uint32_t)s.win[(long long)ioff - wbase] : 255u);
          ioff++;
        }
        nib = (nib << 1) | (uint32_t)y;
        n = 2 * n + 1 + y;
        f = y ? fb : fa;
      }
      // the round's record, kept in registers while the next round's
      // gathers go out
      const bool on_path = recorder && pbits == (nib >> (4 - depth));
      const uint4 rk0 = make_uint4(kk.k[0], kk.k[1], kk.k[2], kk.k[3]);
      const uint4 rk1 = make_uint4(kk.k[4], kk.k[5], kk.k[6], kk.k[7]);
      const uint2 rsv = make_uint2(st[0] | (st[1] << 8) | (st[2] << 16) | (st[3] << 24),
                                   st[4] | (st[5] << 8) | (st[6] << 16) | (st[7] << 24));
      const uint4 rm = make_uint4((uint32_t)(smp[0] & 0xffff) | ((uint32_t)smp[1] << 16),
                                  (uint32_t)(smp[2] & 0xffff) | ((uint32_t)smp[3] << 16),
                                  (uint32_t)(smp[4] & 0xffff) | ((uint32_t)smp[5] << 16),
                                  (uint32_t)(smp[6] & 0xffff) | ((uint32_t)smp[7] << 16));
      const uint32_t rpc = (uint32_t)pr_node | ((uint32_t)cxt << 16) | (((nib >> (3 - depth)) & 1u) << 24);
      cur = (cur << 4) | nib;
      r += 4;
      bool byte_done = false;
      if (r == 8) {
        byte_done = true;
        hist = (hist << 8) | cur;
        cur = 0;
        r = 0;
      }
      if (rd + 1 < nr) gather(kk, st, cur, r, hist);
      // the path's lanes record their bit for the updating warp
      if (on_path) {
        const int i = depth;
        uint4 *k4 = reinterpret_cast<uint4 *>(s.rk + (rd * 4 + i) * kOrders);
        k4[0] = rk0;
        k4[1] = rk1;
        *reinterpret_cast<uint2 *>(s.rs + (rd * 4 + i) * kOrders) = rsv;
        *reinterpret_cast<uint4 *>(s.rsmp + (rd * 4 + i) * kOrders) = rm;
        s.rpc[rd * 4 + i] = rpc;
      }
      if (byte_done) {
        if (lane == 0) s.outb[obyte] = (uint8_t)hist;
        obyte++;
      }
      __syncwarp();
      published++;
      if (lane == 0) {
        __threadfence_block();
        s.prog[0] = published;
      }
    }
    pair_sync(pair);
    dec_unit_end(s, L, tab, slot, t.out + (base >> 3), nunit >> 3, t64);
    pair_sync(pair);
  }
}

// Grid: chunk slots in pairs of warps; warp 2c decodes chunk slot c of the
// CTA, warp 2c + 1 updates its model.
template <bool kLow>
__global__ void __launch_bounds__(kDecMaxPairs * 64)
    decompress_pair_kernel(const ChunkTask *tasks, uint32_t ntasks, uint8_t *slots, uint32_t nslots,
                           const uint8_t *init_tables, const ModelInit *init, uint32_t *queue, uint32_t *status,
                           int unit, uint32_t spin_limit) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  const int pairs = blockDim.x >> 6;
  const DecLayout L = make_dec_layout(unit, pairs, kLow);
  Tables *tab = reinterpret_cast<Tables *>(smem_raw + L.off_tab);
  copy_tables(&g_tables, tab);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int pair = warp >> 1, role = warp & 1;
  const uint32_t gs = blockIdx.x * (uint32_t)pairs + (uint32_t)pair;
  if (gs >= nslots) return;  // both warps of the pair leave together
  const DecSmem s = carve_dec(smem_raw, L, pair);
  uint8_t *slot = slots + (size_t)gs * kSlotTableBytes;
  bool fresh = true;
  for (;;) {
    if (role == 0 && lane == 0) s.prog[1] = atomicAdd(queue, 1u);
    pair_sync(pair);
    const uint32_t ti = s.prog[1];
    pair_sync(pair);
    if (ti >= ntasks) break;
    const ChunkTask t = tasks[ti];
    if (t.unit != (uint32_t)unit || t.cs == 0) {
      if (role == 0 && lane == 0) atomicOr(status, (uint32_t)kDevBadTask);
      continue;
    }
    if (!fresh) {
      uint4 *d = reinterpret_cast<uint4 *>(slot);
      const size_t nv = kSlotTableBytes / 16;
      const int t64 = lane + 32 * role;
      if (init_tables) {
        const uint4 *src = reinterpret_cast<const uint4 *>(init_tables);
        for (size_t i = t64; i < nv; i += 64) d[i] = src[i];
      } else {
        for (size_t i = t64; i < nv; i += 64) d[i] = make_uint4(0, 0, 0, 0);
      }
      pair_sync(pair);
    }
    fresh = false;
    decompress_pair_one<kLow>(t, slot, s, tab, L, init, role, pair, status, spin_limit);
  }
}
