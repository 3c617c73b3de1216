// compress_fast.cuh -- pipelined chunk compressor for units of 32..256 bits.
//
// Included by engine_kernels.cu (shares its tables and coder helpers).
//
// The reference runs five launches per unit and a host round trip between
// them (cucm_compress_v2.cu:1067-1090).  Here one CTA of 7 warps codes a
// chunk, each warp owning one stage, all stages of consecutive units
// overlapped ("tick" t).  The numbers below are roles; compress_fast_one
// gives them to physical warps so that the chain warp has a scheduler to
// itself:
//
//   front warps (3..6, 128 threads)
//     * keys of unit t+2 for all 8 orders (one FNV pass per bit,
//       cucm_compress_v2.cu:723-747), the unit's bits and previous bytes;
//     * slot links of unit t+1: per order, the unit's keys sorted across a
//       warp give every distinct slot of the unit one place (its first
//       position), so every later touch knows it must read the state its
//       predecessor left; a binary search of the previous unit's sorted keys
//       tells whether the slot was touched one unit earlier;
//     * gathers of unit t+1's slot states from the tables in HBM;
//     * stretch, mixer context, mixer output and training of unit t-1
//       (cudamixUnit / cudaupdateMixer, cucm_compress_v2.cu:755-819) against
//       the probabilities as they stand when the previous chain has ended
//       (read from the StateMap records before the chain of unit t-1
//       starts on them).
//   walker warp (2): the bit-history side of the StateMap update for unit
//     t, in bit order, a byte (64 updates) per step: the state each update
//     sees (live), the state each prediction saw (frozen = unit-start value),
//     the next state, written through to the slot table.  It only depends on
//     the bits, never on the probabilities, so it runs a unit ahead of the
//     chain.
//   chain warp (0, lane = order): the StateMap probability updates of unit
//     t-1 in bit order (cucm_compress_v2.cu:592-601); the adaptation rate is
//     carried next to each probability.
//   coder warp (1): the binary arithmetic coder for unit t-2.
//
// After the last data unit the coder keeps coding the stale unit buffer up
// to the chunk end, as cudaencodeUnit does (cucm_compress_v2.cu:850-852).

constexpr int kFastWarps = 7;
constexpr int kFastThreads = kFastWarps * 32;
constexpr int kFastMaxUnit = 256;
constexpr int kWChain = 0, kWCoder = 1, kWWalk = 2, kWFront = 3;
constexpr int kFrontThreads = 128;
constexpr int kSnapThreads = 32 + kFrontThreads;  // chain + front warps (barrier 1)
constexpr int kWinBytes = kFastMaxUnit / 8 + 8;    // input window of a unit (+7 history bytes)

constexpr int kFastStageMin = 2048;

// A compress CTA keeps the whole of the tables in shared memory (reading
// stretch and squash through the read-only cache instead measured 10 %
// slower: the lookups are on the front warps' critical path).
typedef Tables FastTables;

struct FastLayout {
  int U, NSLOT, stage;
  size_t off_tab, off_rec, off_w, off_hk, off_ns, off_key, off_lnk, off_bkt, off_fsw, off_st, off_fr,
      off_yw, off_c1, off_prm, off_win, off_stage, total;
};

__host__ __device__ inline FastLayout make_fast_layout(int U) {
  FastLayout L;
  L.U = U;
  L.NSLOT = U <= 128 ? 128 : 256;  // slots per order and unit: the keys sorted in 4 or 8 per lane
  L.stage = next_pow2(4 * U + 1024);  // a unit codes at most 4U bytes; flushes go out in 512-byte blocks
  if (L.stage < kFastStageMin) L.stage = kFastStageMin;
  const size_t NS = (size_t)L.NSLOT;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    size_t at = o;
    o = (o + bytes + 15) & ~(size_t)15;
    return at;
  };
  L.off_tab = take(sizeof(FastTables));
  L.off_rec = take(sizeof(uint64_t) * kOrders * 256);
  L.off_w = take(sizeof(int32_t) * kMixCtx * kOrders);
  L.off_hk = take(sizeof(uint32_t) * 2 * kOrders * NS);    // keys + 1 by slot, ascending [unit parity][order][slot]
  L.off_ns = take(sizeof(uint16_t) * 2 * kOrders * NS);    // 0x100 | state once written in the unit
  L.off_key = take(sizeof(uint32_t) * 2 * kOrders * U);    // [unit parity][bit][order]
  L.off_lnk = take(sizeof(uint16_t) * 2 * kOrders * U);    // slot + 1 in the previous unit's table, or 0
  L.off_bkt = take(sizeof(uint16_t) * 2 * kOrders * U);    // slot in this unit's table
  L.off_fsw = take((size_t)2 * kOrders * U);               // gathered slot states
  L.off_st = take((size_t)2 * kOrders * U + 4 * kOrders);  // live state (+ the chain's read-ahead)
  L.off_fr = take((size_t)2 * U * kOrders);                // frozen state
  L.off_yw = take(sizeof(uint32_t) * 4 * (U / 32));        // bits, by unit mod 4
  L.off_c1 = take((size_t)4 * (U / 8));                    // previous byte per byte, by unit mod 4
  L.off_prm = take(sizeof(uint16_t) * 2 * U);              // coder input, by unit parity
  L.off_win = take((size_t)kWinBytes);
  L.off_stage = take((size_t)L.stage);
  L.total = o;
  return L;
}

struct FastSmem {
  FastTables *tab;
  uint64_t *rec;     // [256][8]  statep | dt[count] << 32 | dt[count + 1] << 48
  int32_t *w;        // [80*8]
  uint32_t *hk;      // [2][8][NSLOT]
  uint16_t *ns;      // [2][8][NSLOT]
  uint32_t *key;     // [2][U][8]
  uint16_t *lnk;     // [2][U][8]
  uint16_t *bkt;     // [2][U][8]
  uint8_t *fsw;      // [2][U][8]
  uint8_t *st;       // [2][U][8]
  uint8_t *fr;       // [2][U][8]
  uint32_t *yw;      // [4][U/32]
  uint8_t *c1;       // [4][U/8]
  uint16_t *prm;     // [2][U]
  uint8_t *win;      // [kWinBytes]
  uint8_t *stage;
};

__device__ inline FastSmem carve_fast(uint8_t *b, const FastLayout &L) {
  FastSmem s;
  s.tab = reinterpret_cast<FastTables *>(b + L.off_tab);
  s.rec = reinterpret_cast<uint64_t *>(b + L.off_rec);
  s.w = reinterpret_cast<int32_t *>(b + L.off_w);
  s.hk = reinterpret_cast<uint32_t *>(b + L.off_hk);
  s.ns = reinterpret_cast<uint16_t *>(b + L.off_ns);
  s.key = reinterpret_cast<uint32_t *>(b + L.off_key);
  s.lnk = reinterpret_cast<uint16_t *>(b + L.off_lnk);
  s.bkt = reinterpret_cast<uint16_t *>(b + L.off_bkt);
  s.fsw = b + L.off_fsw;
  s.st = b + L.off_st;
  s.fr = b + L.off_fr;
  s.yw = reinterpret_cast<uint32_t *>(b + L.off_yw);
  s.c1 = b + L.off_c1;
  s.prm = reinterpret_cast<uint16_t *>(b + L.off_prm);
  s.win = b + L.off_win;
  s.stage = b + L.off_stage;
  return s;
}

__device__ __forceinline__ void named_barrier(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// Barrier ids: 0 = whole CTA, 1 = chain + front (probabilities read before
// the chain updates them), 2 = front only.
__device__ __forceinline__ void front_sync() { named_barrier(2, kFrontThreads); }

__device__ __forceinline__ int fast_nvalid(uint64_t data_bits, int U, int v) {
  const uint64_t b = (uint64_t)v * U;
  return (v < 0 || b >= data_bits) ? 0 : (int)(data_bits - b < (uint64_t)U ? data_bits - b : (uint64_t)U);
}

// Input byte k of unit v's window: chunk byte v*U/8 - 7 + k, 0 outside
// [0, len).  Thread t < U/8 + 7 loads one byte.
__device__ __forceinline__ uint32_t window_load(const uint8_t *in, uint64_t len, int U, int v, int t) {
  const int64_t i = (int64_t)v * (U / 8) - 7 + t;
  return (t < U / 8 + 7 && i >= 0 && (uint64_t)i < len) ? (uint32_t)__ldg(in + i) : 0u;
}

// Front: keys, bits and previous bytes of unit v from the staged window.
__device__ __forceinline__ void front_keys(const FastSmem &s, const FastLayout &L, int t, int v, int nvalid) {
  const int U = L.U;
  uint32_t *key = s.key + (v & 1) * kOrders * U;
  uint32_t *yw = s.yw + (v & 3) * (U / 32);
  uint8_t *c1 = s.c1 + (v & 3) * (U / 8);
  for (int j0 = 0; j0 < U; j0 += kFrontThreads) {
    const int j = j0 + t;
    uint32_t y = 0;
    if (j < nvalid) {
      const int q = j >> 3, r = j & 7;
      const uint32_t cur = s.win[q + 7];
      const uint32_t h0 = (1u << r) | (cur >> (8 - r));
      const uint32_t p1 = s.win[q + 6];
      uint32_t k8[kOrders];
      uint32_t acc = (kFnvBasis ^ h0) * kFnvPrime;
      k8[0] = h0;
      k8[1] = (p1 << 8) | h0;
      acc = (acc ^ p1) * kFnvPrime;
      CUCM_UNROLL
      for (int o = 2; o < kOrders; o++) {
        acc = (acc ^ (uint32_t)s.win[q + 7 - o]) * kFnvPrime;
        k8[o] = acc & (kSlots - 1);
      }
      uint4 *dst = reinterpret_cast<uint4 *>(key + j * kOrders);
      dst[0] = make_uint4(k8[0], k8[1], k8[2], k8[3]);
      dst[1] = make_uint4(k8[4], k8[5], k8[6], k8[7]);
      y = (cur >> (7 - r)) & 1u;
      if (r == 0) c1[q] = (uint8_t)p1;
    }
    // 32 consecutive bits per warp instruction: pack them.
    const uint32_t word = __ballot_sync(0xffffffffu, y != 0);
    if ((t & 31) == 0 && j < U) yw[j >> 5] = word;
  }
}

// Slot tables: per order and unit, the unit's keys (key + 1) in ascending
// order, padded with kNoKey; a key's slot is the position of its first
// occurrence.  Sorting the unit's keys once replaces a hash table built step
// by step (a claim loop with a shared-memory round trip and a warp barrier
// per two bytes); keeping the repeats in the row (slots with gaps) saves the
// compaction.
constexpr uint32_t kNoKey = 0xffffffffu;

// Ascending bitonic sort of 32 * E values, value p = lane * E + i in a[i]
// of lane `lane`: distances below E are compare-swaps within a lane, the
// others exchange with lane ^ (distance / E) by shuffle.
template <int E>
__device__ __forceinline__ void warp_sort(uint32_t (&a)[E], int lane) {
  constexpr int N = 32 * E;
  CUCM_UNROLL
  for (int k = 2; k <= N; k <<= 1) {
    CUCM_UNROLL
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j >= E) {
        const int lm = j / E;
        const bool lower = (lane & lm) == 0;
        CUCM_UNROLL
        for (int i = 0; i < E; i++) {
          const uint32_t o = __shfl_xor_sync(0xffffffffu, a[i], lm);
          const bool up = ((lane * E + i) & k) == 0;
          a[i] = (up == lower) ? min(a[i], o) : max(a[i], o);
        }
      } else {
        CUCM_UNROLL
        for (int i = 0; i < E; i++) {
          if ((i & j) == 0) {
            const bool up = ((lane * E + i) & k) == 0;
            const uint32_t x = a[i], y = a[i | j];
            a[i] = up ? min(x, y) : max(x, y);
            a[i | j] = up ? max(x, y) : min(x, y);
          }
        }
      }
    }
  }
}

// First position of kp in an ascending row of P (a power of two) entries,
// if it is there: the returned position holds kp exactly when it is present.
template <int P>
__device__ __forceinline__ int row_find(const uint32_t *row, uint32_t kp) {
  int lo = 0;
  CUCM_UNROLL
  for (int step = P >> 1; step > 0; step >>= 1) lo += row[lo + step - 1] < kp ? step : 0;
  return lo;
}

// Front: slots of unit v in its own table, and in the previous unit's.
// Front warp w owns orders 2w and 2w + 1, so no other warp writes their
// rows.  Per order: the unit's keys (bit j = lane + 32 i) are sorted across
// the warp and written in order, then every bit finds its key's first
// position in this unit's row (bkt) and in the previous unit's (lnk =
// position + 1, or 0 when the key was not touched there).  E keys per
// lane: 32 * E >= U, and NSLOT = 32 * E.
template <int E>
__device__ __forceinline__ void front_links(const FastSmem &s, const FastLayout &L, int t, int v, int nvalid) {
  constexpr int P = 32 * E;
  const int U = L.U;
  const uint32_t *key = s.key + (v & 1) * kOrders * U;
  uint16_t *lnk = s.lnk + (v & 1) * kOrders * U;
  uint16_t *bkt = s.bkt + (v & 1) * kOrders * U;
  const int lane = t & 31, w = t >> 5;
  uint32_t kp[2][E], a[2][E];
  CUCM_UNROLL
  for (int h = 0; h < 2; h++) {
    const int o = 2 * w + h;
    CUCM_UNROLL
    for (int i = 0; i < E; i++) {
      const int j = lane + 32 * i;
      kp[h][i] = j < nvalid ? key[j * kOrders + o] + 1 : kNoKey;
      a[h][i] = kp[h][i];
    }
  }
  warp_sort<E>(a[0], lane);
  warp_sort<E>(a[1], lane);
  CUCM_UNROLL
  for (int h = 0; h < 2; h++) {
    uint32_t *row = s.hk + ((v & 1) * kOrders + 2 * w + h) * P;
    CUCM_UNROLL
    for (int i = 0; i < E; i++) row[lane * E + i] = a[h][i];
  }
  __syncwarp();
  CUCM_UNROLL
  for (int h = 0; h < 2; h++) {
    const int o = 2 * w + h;
    const uint32_t *row = s.hk + ((v & 1) * kOrders + o) * P;
    const uint32_t *prow = s.hk + (((v + 1) & 1) * kOrders + o) * P;
    CUCM_UNROLL
    for (int i = 0; i < E; i++) {
      const int j = lane + 32 * i;
      if (j < nvalid) {
        const int d = row_find<P>(row, kp[h][i]);
        const int pd = row_find<P>(prow, kp[h][i]);
        bkt[j * kOrders + o] = (uint16_t)d;
        lnk[j * kOrders + o] = (uint16_t)(prow[pd] == kp[h][i] ? pd + 1 : 0);
      }
    }
  }
}

// Walker: bit-history updates of unit v in bit order, a byte per step.  A
// slot recurs at most once per byte except when two keys of one order
// collide in the 25-bit hash, so the 64 updates of a byte (lane: order
// lane & 7, bits lane >> 3 and (lane >> 3) + 4) are independent and run
// together; a byte with a collision is walked bit by bit instead.  Per
// update: the state it sees (live: an earlier touch in this unit, else the
// frozen unit-start state -- from the previous unit's table when linked),
// the next state, written through to the slot table.  It only depends on
// the bits, never on the probabilities, so it runs a unit ahead of the
// chain.
__device__ __forceinline__ void walk_unit(const FastSmem &s, const FastLayout &L, uint8_t *slot, int lane, int v,
                                          int n) {
  const int U = L.U, NS = L.NSLOT;
  const int o = lane & 7, r0 = lane >> 3;
  const uint32_t *hk = s.hk + ((v & 1) * kOrders + o) * NS;
  const uint16_t *lnk = s.lnk + (v & 1) * U * kOrders;
  const uint16_t *bkt = s.bkt + (v & 1) * U * kOrders;
  const uint8_t *fsb = s.fsw + (v & 1) * U * kOrders;
  const uint32_t *yw = s.yw + (v & 3) * (U / 32);
  uint8_t *st = s.st + (v & 1) * U * kOrders;
  uint8_t *fr = s.fr + (v & 1) * U * kOrders;
  uint16_t *ns_cur = s.ns + ((v & 1) * kOrders + o) * NS;
  const uint16_t *ns_prev = s.ns + (((v + 1) & 1) * kOrders + o) * NS;
  uint8_t *tab = slot + table_offset(o);
  const FastTables *tb = s.tab;
  for (int q = 0; q < (n >> 3); q++) {
    const int ja = q * 8 + r0, jb = ja + 4;
    const int ia = ja * kOrders + o, ib = jb * kOrders + o;
    const uint32_t ba = bkt[ia], bb = bkt[ib];
    // the byte's 8 slots of this order: any two alike?
    bool clash = ba == bb;
CUCM_UNROLL
    for (int k = 0; k < 4; k++) {
      const uint32_t oa = __shfl_sync(0xffffffffu, ba, k * 8 + o);
      const uint32_t ob = __shfl_sync(0xffffffffu, bb, k * 8 + o);
      clash |= (k != r0) && (oa == ba || ob == ba || oa == bb || ob == bb);
    }
    if (!__any_sync(0xffffffffu, clash)) {
      const uint32_t ca = lnk[ia], cb = lnk[ib];
      const uint32_t fa = ca ? (uint32_t)(ns_prev[ca - 1] & 0xffu) : (uint32_t)fsb[ia];
      const uint32_t fb = cb ? (uint32_t)(ns_prev[cb - 1] & 0xffu) : (uint32_t)fsb[ib];
      const uint32_t na = ns_cur[ba], nb = ns_cur[bb];
      const uint32_t ka = hk[ba], kb = hk[bb];
      const uint32_t yword = yw[q >> 2];
      const uint32_t ya = (yword >> (ja & 31)) & 1u, yb = (yword >> (jb & 31)) & 1u;
      const uint32_t la = (na & 0x100u) ? (na & 0xffu) : fa;
      const uint32_t lb = (nb & 0x100u) ? (nb & 0xffu) : fb;
      const uint32_t sa = tb->nex[la][ya], sb = tb->nex[lb][yb];
      ns_cur[ba] = (uint16_t)(0x100u | sa);
      ns_cur[bb] = (uint16_t)(0x100u | sb);
      st[ia] = (uint8_t)la;
      st[ib] = (uint8_t)lb;
      fr[ia] = (uint8_t)fa;
      fr[ib] = (uint8_t)fb;
      tab[ka - 1] = (uint8_t)sa;  // write-through; later touches overwrite it
      tab[kb - 1] = (uint8_t)sb;
    } else if (lane < kOrders) {
      // bit by bit for this byte, lane = order
      for (int r = 0; r < 8; r++) {
        const int j = q * 8 + r, i = j * kOrders + lane;
        const uint32_t b = bkt[i];
        const uint32_t c = lnk[i];
        const uint32_t f = c ? (uint32_t)(ns_prev[c - 1] & 0xffu) : (uint32_t)fsb[i];
        const uint32_t nc = ns_cur[b];
        const uint32_t y = (yw[j >> 5] >> (j & 31)) & 1u;
        const uint32_t lv = (nc & 0x100u) ? (nc & 0xffu) : f;
        const uint32_t ns = tb->nex[lv][y];
        ns_cur[b] = (uint16_t)(0x100u | ns);
        st[i] = (uint8_t)lv;
        fr[i] = (uint8_t)f;
        tab[hk[b] - 1] = (uint8_t)ns;
      }
    }
    __syncwarp();
  }
}

// Chain (lane = order): StateMap probability updates of unit v in bit order.
// A record is statep | dt[c] << 32 | dt[c+1] << 48 for the state's count c;
// the count only ever grows by one per update, so a run of updates of one
// state needs each table value two steps after it is requested.  A step's
// record is loaded two steps ahead; the two results not yet stored when it
// was loaded (the previous step's, stored one step late, and the current
// one) are forwarded from registers, so no shared-memory round trip sits on
// the step-to-step chain.  The bits come 32 to a word; the state three
// steps ahead is read unconditionally (the live-state array has room past
// its end for it).
__device__ __forceinline__ void fast_chain(const FastSmem &s, const FastLayout &L, int o, int v, int n) {
  const int U = L.U;
  const uint8_t *sta = s.st + (v & 1) * U * kOrders + o;
  const uint32_t *yw = s.yw + (v & 3) * (U / 32);
  uint64_t *rec = s.rec + o;  // rec[state * 8 + order]
  const uint16_t *dt = s.tab->dt;
  int st = sta[0];
  int st1 = n > 1 ? sta[kOrders] : 0;
  int st2 = n > 2 ? sta[2 * kOrders] : 0;
  const uint64_t r0 = rec[st * kOrders];
  uint64_t nraw = rec[st1 * kOrders];
  uint32_t val = (uint32_t)r0, d = (uint32_t)(r0 >> 32) & 0xffffu, dn = (uint32_t)(r0 >> 48);
  int pst = st;
  uint32_t pv = val, pd = d, pdn = dn;
  for (int j0 = 0; j0 < n; j0 += 32) {
    uint32_t ywd = yw[j0 >> 5];
    const int je = j0 + 32 < n ? j0 + 32 : n;
    for (int j = j0; j < je; j++) {
      rec[pst * kOrders] = (uint64_t)pv | ((uint64_t)pd << 32) | ((uint64_t)pdn << 48);
      const uint64_t r2 = rec[st2 * kOrders];
      const int st3 = sta[(j + 3) * kOrders];
      const uint32_t y = ywd & 1u;
      ywd >>= 1;
      const uint32_t cnt = val & 1023u;
      const uint32_t dnn = dt[cnt < 1021u ? cnt + 2 : 1023u];
      const int32_t err = (int32_t)((y << 22) - (val >> 10));
      const uint32_t v2 = val + (((uint32_t)(err >> 3) * d) & 0xfffffc00u) + (cnt < 1023u ? 1u : 0u);
      const bool f0 = st1 == st, f1 = st1 == pst;
      const uint32_t nv = f0 ? v2 : f1 ? pv : (uint32_t)nraw;
      const uint32_t nd = f0 ? dn : f1 ? pd : (uint32_t)(nraw >> 32) & 0xffffu;
      const uint32_t ndn = f0 ? dnn : f1 ? pdn : (uint32_t)(nraw >> 48);
      pst = st;
      pv = v2;
      pd = dn;
      pdn = dnn;
      val = nv;
      d = nd;
      dn = ndn;
      nraw = r2;
      st = st1;
      st1 = st2;
      st2 = st3;
    }
  }
  rec[pst * kOrders] = (uint64_t)pv | ((uint64_t)pd << 32) | ((uint64_t)pdn << 48);
}

// Front: stretched probabilities of unit v's bits (thread t: bits t and
// t + 128) as the records stand when the previous chain has ended, read
// before the chain of unit v changes them.
__device__ __forceinline__ void front_probs(const FastSmem &s, const FastLayout &L, int t, int v, int nvalid,
                                            int (&smps)[2][kOrders]) {
  const int U = L.U;
  const uint8_t *fr = s.fr + (v & 1) * U * kOrders;
  CUCM_UNROLL
  for (int h = 0; h < 2; h++) {
    const int j = t + h * kFrontThreads;
    if (j < U && j < nvalid) {
      const uint64_t f8 = *reinterpret_cast<const uint64_t *>(fr + j * kOrders);
      CUCM_UNROLL
      for (int o = 0; o < kOrders; o++) {
        const uint32_t stt = (uint32_t)(f8 >> (8 * o)) & 0xffu;
        smps[h][o] = s.tab->stretch[reinterpret_cast<const uint32_t *>(s.rec)[2 * (stt * kOrders + o)] >> 20];
      }
    }
  }
}

// Front: predictions, mixer output and training of unit v from the
// probabilities front_probs read; thread t handles bits t and t + 128.
__device__ __forceinline__ void front_mix(const FastSmem &s, const FastLayout &L, int t, int v, int nvalid,
                                          int (&smps)[2][kOrders]) {
  const int U = L.U;
  const uint32_t *yw = s.yw + (v & 3) * (U / 32);
  const uint8_t *c1 = s.c1 + (v & 3) * (U / 8);
  uint16_t *prm = s.prm + (v & 1) * U;
  const uint16_t *prm_old = s.prm + ((v + 1) & 1) * U;
  int cxs[2] = {0, 0}, errs[2] = {0, 0};
  bool has[2] = {false, false};
  CUCM_UNROLL
  for (int h = 0; h < 2; h++) {
    const int j = t + h * kFrontThreads;
    if (j < U) {
      if (j < nvalid) {
        int olen = 0;
        CUCM_UNROLL
        for (int o = 0; o < kOrders; o++) olen += (smps[h][o] != 1);
        const int cx = olen + (c1[j >> 3] >> 5) * 10;
        const int pr = mix_pr(s.w, cx, smps[h], s.tab);
        const int y = (yw[j >> 5] >> (j & 31)) & 1;
        prm[j] = (uint16_t)((pr << 1) | y);
        cxs[h] = cx;
        errs[h] = ((y << 12) - pr) * 7;
        has[h] = true;
      } else {
        prm[j] = prm_old[j];  // stale entry, re-coded as the reference does
      }
    }
  }
  front_sync();  // every weight read before any update
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

// Front: table words holding the slot states of unit v, into registers.
// Each thread takes entries e = t + 128 i (i < GR) of the [8][U] grid; GR is
// 8 for units up to 128 bits and 16 up to 256.
template <int GR>
__device__ __forceinline__ void front_gather(const FastSmem &s, const FastLayout &L, const uint8_t *slot, int t,
                                             int v, int nvalid, uint32_t g[GR]) {
  const int U = L.U;
  const uint32_t *key = s.key + (v & 1) * kOrders * U;
  CUCM_UNROLL
  for (int i = 0; i < GR; i++) {
    const int e = t + i * kFrontThreads;
    if (e < kOrders * U) {
      const int j = e >> 3, o = e & 7;
      if (j < nvalid) {
        const uint32_t k = key[e];
        const uint32_t *p = reinterpret_cast<const uint32_t *>(slot + table_offset(o) + (k & ~3u));
        g[i] = __ldcg(p);
      }
    }
  }
}

template <int GR>
__device__ __forceinline__ void front_store_gather(const FastSmem &s, const FastLayout &L, int t, int v,
                                                   const uint32_t g[GR]) {
  const int U = L.U;
  const uint32_t *key = s.key + (v & 1) * kOrders * U;
  uint8_t *fsb = s.fsw + (v & 1) * kOrders * U;
  CUCM_UNROLL
  for (int i = 0; i < GR; i++) {
    const int e = t + i * kFrontThreads;
    if (e < kOrders * U) fsb[e] = (uint8_t)(g[i] >> (8 * (key[e] & 3)));
  }
}

constexpr uint64_t kTailOffloadBits = 4096;  // shorter stale tails are coded in place

template <int GR>
__device__ void compress_fast_one(const ChunkTask &t, uint8_t *slot, const FastSmem &s, const FastLayout &L,
                                  const ModelInit *init, uint32_t *status, TailTask *tails, uint32_t *tail_count) {
  const int tid = threadIdx.x;
  const int pw = tid >> 5, lane = tid & 31;
  // Role of each warp.  A CTA's warp i issues from the SM's scheduler i % 4,
  // so warp 3 (alone on its scheduler) takes the chain, the slowest role;
  // the coder shares a scheduler with the walker, the front warps pair up
  // (measured 795 -> 753 ms per 256 MiB launch against roles in warp order).
  const int warp = (int)((0x6250413u >> (4 * pw)) & 15u);
  const int U = L.U;
  const uint64_t len = t.in_len < t.cs ? t.in_len : t.cs;
  const uint64_t total_bits = 8ull * t.cs;
  const uint64_t data_bits = 8ull * len;
  const int nU = (int)((data_bits + U - 1) / U);
  const bool front = warp >= kWFront;
  const int ft = (warp - kWFront) * 32 + lane;
  auto ncode_of = [&](int v) -> int {
    const uint64_t b = (uint64_t)v * U;
    return b >= total_bits ? 0 : (int)(total_bits - b < (uint64_t)U ? total_bits - b : (uint64_t)U);
  };

  for (int i = tid; i < kOrders * 256; i += blockDim.x) {
    const uint32_t v = init->statep[i & 7][i >> 3];  // rec[state * 8 + order]
    const uint32_t c = v & 1023u;
    s.rec[i] = (uint64_t)v | ((uint64_t)s.tab->dt[c] << 32) | ((uint64_t)s.tab->dt[c < 1023u ? c + 1 : 1023u] << 48);
  }
  for (int i = tid; i < kMixCtx * kOrders; i += blockDim.x) s.w[i] = init->w[i];
  for (int i = tid; i < 2 * U; i += blockDim.x) s.prm[i] = 0;  // cucm_compress_v2.cu:1039-1040
  for (int i = tid; i < 2 * kOrders * L.NSLOT; i += blockDim.x) s.hk[i] = 0;

  Coder c{0u, 0xffffffffu, 0, 0};
  uint32_t g[GR];
  uint32_t wbyte = 0;
  __syncthreads();

  // Prologue: keys of units 0 and 1, links and gathers of unit 0.
  if (front) {
    for (int v = 0; v < 2 && v < nU; v++) {
      const uint32_t b = window_load(t.in, len, U, v, ft);
      if (ft < U / 8 + 7) s.win[ft] = (uint8_t)b;
      front_sync();
      front_keys(s, L, ft, v, fast_nvalid(data_bits, U, v));
      front_sync();
    }
    front_links<GR / 2>(s, L, ft, 0, fast_nvalid(data_bits, U, 0));
    front_gather<GR>(s, L, slot, ft, 0, fast_nvalid(data_bits, U, 0), g);
    front_store_gather<GR>(s, L, ft, 0, g);
    if (nU > 2) wbyte = window_load(t.in, len, U, 2, ft);
  }
  __syncthreads();

  for (int tau = 0; tau < nU + 2; tau++) {
    const int um = tau - 1;
    // gathers of unit tau+1 go out first; they land while the front works
    const int nv1 = fast_nvalid(data_bits, U, tau + 1);
    if (front && tau + 1 < nU) front_gather<GR>(s, L, slot, ft, tau + 1, nv1, g);
    int smps[2][kOrders];
    if (warp == kWChain || front) {
      if (front && um >= 0 && um < nU) front_probs(s, L, ft, um, fast_nvalid(data_bits, U, um), smps);
      named_barrier(1, kSnapThreads);
    }
    if (warp == kWChain) {
      if (um >= 0 && um < nU && lane < kOrders) fast_chain(s, L, lane, um, fast_nvalid(data_bits, U, um));
    } else if (warp == kWCoder) {
      const int uc = tau - 2;
      if (uc >= 0 && uc < nU) {
        coder_run_p(c, s.prm + (uc & 1) * U, s.stage, L.stage, ncode_of(uc));
        coder_flush_p(c, s.stage, L.stage, t.out, t.out_cap);
      }
    } else if (warp == kWWalk) {
      if (tau < nU) {
        uint4 *z4 = reinterpret_cast<uint4 *>(s.ns + (tau & 1) * kOrders * L.NSLOT);
        for (int i = lane; i < kOrders * L.NSLOT / 8; i += 32) z4[i] = make_uint4(0, 0, 0, 0);
        __syncwarp();
        walk_unit(s, L, slot, lane, tau, fast_nvalid(data_bits, U, tau));
      }
    } else {
      if (um >= 0 && um < nU) front_mix(s, L, ft, um, fast_nvalid(data_bits, U, um), smps);
      if (tau + 1 < nU) {
        front_links<GR / 2>(s, L, ft, tau + 1, nv1);
        if (tau + 2 < nU) {
          if (ft < U / 8 + 7) s.win[ft] = (uint8_t)wbyte;
          front_sync();
          front_keys(s, L, ft, tau + 2, fast_nvalid(data_bits, U, tau + 2));
          if (tau + 3 < nU) wbyte = window_load(t.in, len, U, tau + 3, ft);
        }
        front_store_gather<GR>(s, L, ft, tau + 1, g);
      }
    }
    __syncthreads();
  }

  if (warp == kWCoder) {
    const uint16_t *last = s.prm + ((nU - 1) & 1) * U;
    const uint64_t coded = (uint64_t)nU * U;
    const uint64_t left = total_bits > coded ? total_bits - coded : 0;
    if (tails && left >= kTailOffloadBits) {
      // the stale tail goes to the tail pass: the ring drains to the
      // payload, the coder state and the unit buffer to a tail task, and the
      // CTA moves on to its next chunk
      const uint32_t mask = (uint32_t)L.stage - 1;
      for (uint64_t i = c.flushed + lane; i < c.head; i += 32)
        if (i < t.out_cap) t.out[i] = s.stage[(uint32_t)i & mask];
      uint32_t k = 0;
      if (lane == 0) k = atomicAdd(tail_count, 1u);
      k = __shfl_sync(0xffffffffu, k, 0);
      TailTask &T = tails[k];
      for (int j = lane; j < U; j += 32) T.prm[j] = last[j];
      if (lane == 0) {
        T.out = t.out;
        T.cap = t.out_cap;
        T.result = t.result;
        T.head = c.head;
        T.bits = left;
        T.x1 = c.x1;
        T.x2 = c.x2;
        T.unit = (uint32_t)U;
      }
      __syncwarp();
    } else {
      for (int v = nU;; v++) {
        const int n = ncode_of(v);
        if (n <= 0) break;
        coder_run_p(c, last, s.stage, L.stage, n);
        coder_flush_p(c, s.stage, L.stage, t.out, t.out_cap);
      }
      coder_finish_p(c, s.stage, L.stage, t.out, t.out_cap, t.result);
      if (lane == 0 && c.head > t.out_cap) atomicOr(status, (uint32_t)kDevOverflow);
    }
  }
  __syncthreads();
}

// Persistent CTA: chunks from the work queue, one after the other, each in
// this CTA's slot tables (restored to the initial model between chunks).
template <int GR>
__device__ __forceinline__ void compress_fast_loop(const ChunkTask *tasks, uint32_t ntasks, uint8_t *slots,
                                                   const uint8_t *init_tables, const ModelInit *init,
                                                   uint32_t *queue, uint32_t *status, int unit, TailTask *tails,
                                                   uint32_t *tail_count) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  const FastLayout L = make_fast_layout(unit);
  const FastSmem s = carve_fast(smem_raw, L);
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
    compress_fast_one<GR>(t, slot, s, L, init, status, tails, tail_count);
  }
}

// Units up to 128 bits.  (Capping the registers at 96 so that three CTAs
// share an SM made each CTA 35-44 % slower: more CTAs did not pay for it.)
__global__ void __launch_bounds__(kFastThreads, 2)
    compress_fast_kernel(const ChunkTask *tasks, uint32_t ntasks, uint8_t *slots, const uint8_t *init_tables,
                         const ModelInit *init, uint32_t *queue, uint32_t *status, int unit, TailTask *tails,
                         uint32_t *tail_count) {
  compress_fast_loop<8>(tasks, ntasks, slots, init_tables, init, queue, status, unit, tails, tail_count);
}

// Units of 160..256 bits.
__global__ void __launch_bounds__(kFastThreads, 2)
    compress_fast_kernel_wide(const ChunkTask *tasks, uint32_t ntasks, uint8_t *slots, const uint8_t *init_tables,
                              const ModelInit *init, uint32_t *queue, uint32_t *status, int unit, TailTask *tails,
                              uint32_t *tail_count) {
  compress_fast_loop<16>(tasks, ntasks, slots, init_tables, init, queue, status, unit, tails, tail_count);
}

// One chunk, task passed by value, tables at `slot` (no work queue); the
// stale tail is coded in place.
template <int GR>
__global__ void __launch_bounds__(kFastThreads, 2)
    compress_fast_single_kernel(const ChunkTask t, uint8_t *slot, const ModelInit *init, uint32_t *status) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  const FastLayout L = make_fast_layout((int)t.unit);
  const FastSmem s = carve_fast(smem_raw, L);
  copy_tables(&g_tables, s.tab);
  __syncthreads();
  compress_fast_one<GR>(t, slot, s, L, init, status, nullptr, nullptr);
}

// The tail pass: one thread per handed-over chunk codes its stale tail (the
// unit buffer again and again up to the chunk end), writes the bytes, the
// flush byte (cucm_compress_v2.cu:902) and the payload length.  Same coder
// step as coder_step; the buffer is read through the read-only cache, four
// entries per load.
__global__ void __launch_bounds__(128) compress_tail_kernel(const TailTask *tails, const uint32_t *count,
                                                            uint32_t *status) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *count) return;
  const TailTask &T = tails[i];
  uint32_t x1 = T.x1, x2 = T.x2;
  uint64_t head = T.head;
  const uint64_t cap = T.cap;
  uint8_t *out = T.out;
  const uint32_t U = T.unit;
  const uint64_t *prm4 = reinterpret_cast<const uint64_t *>(T.prm);
  uint64_t left = T.bits;
  uint32_t j4 = 0;  // next group of four entries
  while (left) {
    const uint64_t e4 = __ldg(prm4 + j4);
    j4 = (4 * (j4 + 1) == U) ? 0u : j4 + 1;
    const int n = left < 4 ? (int)left : 4;
    left -= (uint64_t)n;
CUCM_UNROLL
    for (int q = 0; q < 4; q++) {
      if (q < n) {
        const uint32_t e = (uint32_t)(e4 >> (16 * q)) & 0xffffu;
        const uint32_t xm = x1 + __umulhi(x2 - x1, (e >> 1) << 20);
        if (e & 1) x2 = xm; else x1 = xm + 1;
        while ((x1 ^ x2) < 0x1000000u) {
          if (head < cap) out[head] = (uint8_t)(x2 >> 24);
          head++;
          x1 <<= 8;
          x2 = (x2 << 8) | 255u;
        }
      }
    }
  }
  if (head < cap) out[head] = (uint8_t)(x1 >> 24);
  head++;
  *T.result = head;
  if (head > cap) atomicOr(status, (uint32_t)kDevOverflow);
}
