/*
 * cucm_oracle.c -- CPU restatement of CuCM's chunked context-mixing coder.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA product, never part of
 * it.  Parity of this file with the reference is pinned by
 * tests/test_oracle.py (reference binaries built from the reference's own
 * sources by oracle/make_ref.py, plus committed golden fixtures).
 *
 * Model (cucm_compress_v2.cu:551-705):
 *   8 StateMaps, order o = 0..7, each with 2^25 one-byte bit-history slots
 *   and 256 adaptive 32-bit probabilities (22-bit p, 10-bit count), keyed by
 *   an FNV-1 hash of the partial current byte and the o previous bytes;
 *   one Mixer of 80 contexts x 8 int32 weights; a 32-bit carry-less binary
 *   arithmetic coder with 12-bit probabilities.
 *
 * The chunk coder follows the reference's GPU schedule, not lpaq's
 * bit-serial one: within a "unit" of `unit` bits every prediction uses the
 * model as it was at the unit start; the Mixer deltas and the StateMap
 * updates of the unit are applied after the unit has been coded.
 */
#include "cucm_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* cucm_compress_v2.cu:35-285 (identical copy at cucm_decompress_v2.cu:16-266).
 * Row s holds the next bit-history state after coding a 0 and a 1. */
static const uint8_t kNextState[256][2] = {
    {  1,  2}, {  3,  5}, {  4,  6}, {  7, 10}, {  8, 12}, {  9, 13}, { 11, 14}, { 15, 19},
    { 16, 23}, { 17, 24}, { 18, 25}, { 20, 27}, { 21, 28}, { 22, 29}, { 26, 30}, { 31, 33},
    { 32, 35}, { 32, 35}, { 32, 35}, { 32, 35}, { 34, 37}, { 34, 37}, { 34, 37}, { 34, 37},
    { 34, 37}, { 34, 37}, { 36, 39}, { 36, 39}, { 36, 39}, { 36, 39}, { 38, 40}, { 41, 43},
    { 42, 45}, { 42, 45}, { 44, 47}, { 44, 47}, { 46, 49}, { 46, 49}, { 48, 51}, { 48, 51},
    { 50, 52}, { 53, 43}, { 54, 57}, { 54, 57}, { 56, 59}, { 56, 59}, { 58, 61}, { 58, 61},
    { 60, 63}, { 60, 63}, { 62, 65}, { 62, 65}, { 50, 66}, { 67, 55}, { 68, 57}, { 68, 57},
    { 70, 73}, { 70, 73}, { 72, 75}, { 72, 75}, { 74, 77}, { 74, 77}, { 76, 79}, { 76, 79},
    { 62, 81}, { 62, 81}, { 64, 82}, { 83, 69}, { 84, 71}, { 84, 71}, { 86, 73}, { 86, 73},
    { 44, 59}, { 44, 59}, { 58, 61}, { 58, 61}, { 60, 49}, { 60, 49}, { 76, 89}, { 76, 89},
    { 78, 91}, { 78, 91}, { 80, 92}, { 93, 69}, { 94, 87}, { 94, 87}, { 96, 45}, { 96, 45},
    { 48, 99}, { 48, 99}, { 88,101}, { 88,101}, { 80,102}, {103, 69}, {104, 87}, {104, 87},
    {106, 57}, {106, 57}, { 62,109}, { 62,109}, { 88,111}, { 88,111}, { 80,112}, {113, 85},
    {114, 87}, {114, 87}, {116, 57}, {116, 57}, { 62,119}, { 62,119}, { 88,121}, { 88,121},
    { 90,122}, {123, 85}, {124, 97}, {124, 97}, {126, 57}, {126, 57}, { 62,129}, { 62,129},
    { 98,131}, { 98,131}, { 90,132}, {133, 85}, {134, 97}, {134, 97}, {136, 57}, {136, 57},
    { 62,139}, { 62,139}, { 98,141}, { 98,141}, { 90,142}, {143, 95}, {144, 97}, {144, 97},
    { 68, 57}, { 68, 57}, { 62, 81}, { 62, 81}, { 98,147}, { 98,147}, {100,148}, {149, 95},
    {150,107}, {150,107}, {108,151}, {108,151}, {100,152}, {153, 95}, {154,107}, {108,155},
    {100,156}, {157, 95}, {158,107}, {108,159}, {100,160}, {161,105}, {162,107}, {108,163},
    {110,164}, {165,105}, {166,117}, {118,167}, {110,168}, {169,105}, {170,117}, {118,171},
    {110,172}, {173,105}, {174,117}, {118,175}, {110,176}, {177,105}, {178,117}, {118,179},
    {110,180}, {181,115}, {182,117}, {118,183}, {120,184}, {185,115}, {186,127}, {128,187},
    {120,188}, {189,115}, {190,127}, {128,191}, {120,192}, {193,115}, {194,127}, {128,195},
    {120,196}, {197,115}, {198,127}, {128,199}, {120,200}, {201,115}, {202,127}, {128,203},
    {120,204}, {205,115}, {206,127}, {128,207}, {120,208}, {209,125}, {210,127}, {128,211},
    {130,212}, {213,125}, {214,137}, {138,215}, {130,216}, {217,125}, {218,137}, {138,219},
    {130,220}, {221,125}, {222,137}, {138,223}, {130,224}, {225,125}, {226,137}, {138,227},
    {130,228}, {229,125}, {230,137}, {138,231}, {130,232}, {233,125}, {234,137}, {138,235},
    {130,236}, {237,125}, {238,137}, {138,239}, {130,240}, {241,125}, {242,137}, {138,243},
    {130,244}, {245,135}, {246,137}, {138,247}, {140,248}, {249,135}, {250, 69}, { 80,251},
    {140,252}, {249,135}, {250, 69}, { 80,251}, {140,252}, {  0,  0}, {  0,  0}, {  0,  0},
};

const uint8_t *co_next_state_table(void) { return &kNextState[0][0]; }

static int32_t g_squash[4096], g_stretch[4096], g_dt[1024];
static pthread_once_t g_once = PTHREAD_ONCE_INIT;

/* cucm_compress_v2.cu:681-705: squash by linear interpolation between 33
 * knots spaced 128 apart, stretch as its inverse, dt[i] = 16384/(2i+3). */
static void build_tables(void) {
  static const int knots[33] = {1,    2,    3,    6,    10,   16,   27,   45,   73,   120,  194,
                                310,  488,  747,  1101, 1546, 2047, 2549, 2994, 3348, 3607, 3785,
                                3901, 3975, 4022, 4050, 4068, 4079, 4085, 4089, 4092, 4093, 4094};
  for (int k = 0; k <= 4094; k++) {
    int d = k - 2047;
    int frac = d & 127;
    int seg = (d >> 7) + 16;
    g_squash[k] = (knots[seg] * (128 - frac) + knots[seg + 1] * frac + 64) >> 7;
  }
  g_squash[4095] = 4095;
  int next = 0;
  for (int x = -2047; x <= 2047; x++) {
    int v = g_squash[x + 2047];
    for (int j = next; j <= v; j++) g_stretch[j] = x;
    next = v + 1;
  }
  g_stretch[4095] = 2047;
  for (int i = 0; i < 1024; i++) g_dt[i] = 16384 / (i + i + 3);
}

static void tables_once(void) { pthread_once(&g_once, build_tables); }

void co_tables(int32_t squash[4096], int32_t stretch[4096], int32_t dt[1024]) {
  tables_once();
  memcpy(squash, g_squash, sizeof g_squash);
  memcpy(stretch, g_stretch, sizeof g_stretch);
  memcpy(dt, g_dt, sizeof g_dt);
}

co_model *co_model_new(void) {
  tables_once();
  co_model *m = (co_model *)calloc(1, sizeof(co_model));
  if (!m) return NULL;
  m->states = (uint8_t *)calloc((size_t)CO_ORDERS * CO_SLOTS, 1);
  if (!m->states) {
    free(m);
    return NULL;
  }
  for (int o = 0; o < CO_ORDERS; o++)
    for (int s = 0; s < 256; s++) m->statep[o][s] = 1u << 31; /* cucm_compress_v2.cu:565 */
  return m;
}

void co_model_free(co_model *m) {
  if (!m) return;
  free(m->states);
  free(m);
}

void co_model_copy(co_model *dst, const co_model *src) {
  memcpy(dst->states, src->states, (size_t)CO_ORDERS * CO_SLOTS);
  memcpy(dst->statep, src->statep, sizeof dst->statep);
  memcpy(dst->w, src->w, sizeof dst->w);
}

/* ---- model primitives --------------------------------------------------- */

/* Context hashes of one bit (cucm_compress_v2.cu:723-747): h[0] is the
 * partial current byte with a leading 1 at bit `bit`; h[i] (i >= 1) the i-th
 * previous byte, 0 before the start of the buffer.  Order o hashes
 * h[0..o] with FNV-1 (offset 2166136261, prime 16777619) and keeps 25 bits.
 * Only the low 25 bits survive, so 32-bit arithmetic is exact. */
static inline void bit_hashes(const uint8_t *buf, size_t byte, int bit, uint32_t hs[CO_ORDERS]) {
  uint32_t h0 = (1u << bit) | ((uint32_t)buf[byte] >> (8 - bit));
  uint32_t acc = 2166136261u;
  acc = (acc ^ h0) * 16777619u;
  hs[0] = acc & 0x1ffffffu;
  for (int o = 1; o < CO_ORDERS; o++) {
    uint32_t prev = (byte >= (size_t)o) ? buf[byte - o] : 0u;
    acc = (acc ^ prev) * 16777619u;
    hs[o] = acc & 0x1ffffffu;
  }
}

/* StateMap::update (cucm_compress_v2.cu:592-601), with the reference's int
 * conversions written out as 32-bit wrapping arithmetic. */
static inline void sm_update(uint8_t *states, uint32_t *statep, uint32_t slot, int y) {
  int s = states[slot];
  uint32_t v = statep[s];
  uint32_t cnt = v & 1023u;
  int32_t err = (int32_t)(((uint32_t)y << 22) - (v >> 10));
  uint32_t adj = ((uint32_t)(err >> 3) * (uint32_t)g_dt[cnt]) & 0xfffffc00u;
  v += adj;
  if (cnt < 1023) v++;
  statep[s] = v;
  states[slot] = kNextState[s][y];
}

/* Mixer::p (cucm_compress_v2.cu:636-644) plus the caller's `if (pr < 2048)
 * pr++` (cucm_compress_v2.cu:785-786). */
static inline int mixer_pr(const int32_t *w, int cxt, const int smp[CO_ORDERS]) {
  int64_t sum = 0;
  for (int i = 0; i < CO_ORDERS; i++) sum += (int64_t)w[cxt * CO_ORDERS + i] * smp[i];
  sum >>= 16;
  int idx = sum < -2047 ? -2047 : (sum > 2048 ? 2048 : (int)sum);
  int pr = g_squash[idx + 2047];
  if (pr < 2048) pr++;
  return pr;
}

/* Mixer::update (cucm_compress_v2.cu:663-678); int adds wrap like atomicAdd. */
static inline void mixer_update(int32_t *w, int cxt, const int smp[CO_ORDERS], int y, int pr) {
  int err = ((y << 12) - pr) * 7;
  for (int i = 0; i < CO_ORDERS; i++) {
    int32_t d = (int32_t)(((int64_t)err * smp[i]) >> 16);
    w[cxt * CO_ORDERS + i] = (int32_t)((uint32_t)w[cxt * CO_ORDERS + i] + (uint32_t)d);
  }
}

/* Mixer context (cucm_compress_v2.cu:775-784): number of orders whose
 * stretched prediction is not 1, plus 10 * (previous byte >> 5). */
static inline int mixer_cxt(const int smp[CO_ORDERS], int c1) {
  int olen = 0;
  for (int i = 0; i < CO_ORDERS; i++) olen += (smp[i] != 1);
  return olen + (c1 >> 5) * 10;
}

/* Binary arithmetic coder step (cucm_compress_v2.cu:855-862). */
static inline uint32_t coder_mid(uint32_t x1, uint32_t x2, int pr) {
  uint32_t r = x2 - x1;
  return x1 + (r >> 12) * (uint32_t)pr + (((r & 0xfffu) * (uint32_t)pr) >> 12);
}

/* ---- host prelearn (bit-serial, no unit freezing) ----------------------- */

/* One bit of the host prelearn model: predict, then update mixer and all
 * StateMaps (cucm_compress_v2.cu:930-968). */
static inline int prelearn_bit(co_model *m, const uint8_t *buf, size_t pos, int y_known, int *pr_out,
                               uint32_t hs[CO_ORDERS], int smp[CO_ORDERS], int *cxt_out) {
  size_t byte = pos >> 3;
  int bit = (int)(pos & 7);
  bit_hashes(buf, byte, bit, hs);
  for (int o = 0; o < CO_ORDERS; o++) {
    uint8_t s = m->states[(size_t)o * CO_SLOTS + hs[o]];
    smp[o] = g_stretch[m->statep[o][s] >> 20];
  }
  int c1 = byte >= 1 ? buf[byte - 1] : 0;
  int cxt = mixer_cxt(smp, c1);
  *pr_out = mixer_pr(m->w, cxt, smp);
  *cxt_out = cxt;
  return y_known;
}

static inline void prelearn_update(co_model *m, const uint32_t hs[CO_ORDERS], const int smp[CO_ORDERS],
                                   int cxt, int y, int pr) {
  mixer_update(m->w, cxt, smp, y, pr);
  for (int o = 0; o < CO_ORDERS; o++)
    sm_update(m->states + (size_t)o * CO_SLOTS, m->statep[o], hs[o], y);
}

size_t co_prelearn_encode(co_model *m, const uint8_t *in, size_t n, uint8_t *out, size_t cap) {
  tables_once();
  uint32_t x1 = 0, x2 = 0xffffffffu;
  size_t off = 0;
  uint32_t hs[CO_ORDERS];
  int smp[CO_ORDERS], pr, cxt;
  for (size_t pos = 0; pos < n * 8; pos++) {
    int y = (in[pos >> 3] >> (7 - (pos & 7))) & 1;
    prelearn_bit(m, in, pos, y, &pr, hs, smp, &cxt);
    prelearn_update(m, hs, smp, cxt, y, pr);
    uint32_t xmid = coder_mid(x1, x2, pr);
    if (y) x2 = xmid; else x1 = xmid + 1;
    while (((x1 ^ x2) & 0xff000000u) == 0) {
      if (off >= cap) return (size_t)-1;
      out[off++] = (uint8_t)(x2 >> 24);
      x1 <<= 8;
      x2 = (x2 << 8) | 255u;
    }
  }
  if (off >= cap) return (size_t)-1;
  out[off++] = (uint8_t)(x1 >> 24); /* cucm_compress_v2.cu:978-979 */
  return off;
}

void co_prelearn_train(co_model *m, const uint8_t *in, size_t n) {
  tables_once();
  uint32_t hs[CO_ORDERS];
  int smp[CO_ORDERS], pr, cxt;
  for (size_t pos = 0; pos < n * 8; pos++) {
    int y = (in[pos >> 3] >> (7 - (pos & 7))) & 1;
    prelearn_bit(m, in, pos, y, &pr, hs, smp, &cxt);
    prelearn_update(m, hs, smp, cxt, y, pr);
  }
}

void co_prelearn_decode(co_model *m, const uint8_t *in, size_t in_n, uint8_t *out, size_t n) {
  tables_once();
  memset(out, 0, n);
  uint32_t x1 = 0, x2 = 0xffffffffu, x = 0;
  size_t ioff = 0;
  for (int i = 0; i < 4; i++) x = (x << 8) | (ioff < in_n ? in[ioff++] : 255u);
  uint32_t hs[CO_ORDERS];
  int smp[CO_ORDERS], pr, cxt;
  for (size_t pos = 0; pos < n * 8; pos++) {
    prelearn_bit(m, out, pos, 0, &pr, hs, smp, &cxt);
    uint32_t xmid = coder_mid(x1, x2, pr);
    int y = x <= xmid;
    if (y) x2 = xmid; else x1 = xmid + 1;
    prelearn_update(m, hs, smp, cxt, y, pr);
    while (((x1 ^ x2) & 0xff000000u) == 0) {
      x1 <<= 8;
      x2 = (x2 << 8) | 255u;
      x = (x << 8) | (ioff < in_n ? in[ioff++] : 255u);
    }
    out[pos >> 3] |= (uint8_t)(y << (7 - (pos & 7)));
  }
}

/* ---- unit-frozen chunk coder -------------------------------------------- */

typedef struct unit_buf {
  int unit;
  uint32_t *hash;  /* [CO_ORDERS][unit] */
  int *smp;        /* [CO_ORDERS][unit] */
  int *cxt;        /* [unit] */
  int *pr;         /* [unit] */
  int *y;          /* [unit] */
  uint16_t *prm;   /* [unit] encoder input pr<<1|y, persists across units */
} unit_buf;

static int unit_buf_init(unit_buf *u, int unit) {
  u->unit = unit;
  u->hash = (uint32_t *)calloc((size_t)CO_ORDERS * unit, sizeof(uint32_t));
  u->smp = (int *)calloc((size_t)CO_ORDERS * unit, sizeof(int));
  u->cxt = (int *)calloc(unit, sizeof(int));
  u->pr = (int *)calloc(unit, sizeof(int));
  u->y = (int *)calloc(unit, sizeof(int));
  u->prm = (uint16_t *)calloc(unit, sizeof(uint16_t));
  return (u->hash && u->smp && u->cxt && u->pr && u->y && u->prm) ? 0 : -1;
}

static void unit_buf_free(unit_buf *u) {
  free(u->hash);
  free(u->smp);
  free(u->cxt);
  free(u->pr);
  free(u->y);
  free(u->prm);
}

/* Predict + mix every bit of unit `u` with the frozen model
 * (cudapredictUnit cucm_compress_v2.cu:711-750, cudamixUnit 755-792).  Bit
 * b of the chunk is processed when b < 8*len (input bound) and b < 8*cs
 * (chunk bound).  Returns the number of such bits (a prefix of the unit). */
static int unit_predict(const co_model *m, const uint8_t *chunk, size_t len, size_t cs, uint64_t base,
                        unit_buf *ub) {
  int nvalid = 0;
  for (int j = 0; j < ub->unit; j++) {
    uint64_t b = base + (uint64_t)j;
    if (b >= 8 * (uint64_t)len || b >= 8 * (uint64_t)cs) break;
    size_t byte = (size_t)(b >> 3);
    int bit = (int)(b & 7);
    uint32_t hs[CO_ORDERS];
    bit_hashes(chunk, byte, bit, hs);
    int smp[CO_ORDERS];
    for (int o = 0; o < CO_ORDERS; o++) {
      uint8_t s = m->states[(size_t)o * CO_SLOTS + hs[o]];
      smp[o] = g_stretch[m->statep[o][s] >> 20];
      ub->hash[o * ub->unit + j] = hs[o];
      ub->smp[o * ub->unit + j] = smp[o];
    }
    int c1 = byte >= 1 ? chunk[byte - 1] : 0;
    int cxt = mixer_cxt(smp, c1);
    int pr = mixer_pr(m->w, cxt, smp);
    int y = (chunk[byte] >> (7 - bit)) & 1;
    ub->cxt[j] = cxt;
    ub->pr[j] = pr;
    ub->y[j] = y;
    ub->prm[j] = (uint16_t)((pr << 1) | y);
    nvalid++;
  }
  return nvalid;
}

/* Deferred updates of one unit (cudaupdateMixer cucm_compress_v2.cu:794-819,
 * cudaStateMapUpdate 821-839; decoder updateStateMap/updateMixer
 * cucm_decompress_v2.cu:870-896).  The mixer deltas depend only on
 * unit-start values, so applying them in bit order equals the reference's
 * atomicAdd sum.  StateMap updates run in bit order per order and read the
 * live slot, i.e. after earlier same-slot updates of the unit. */
static void unit_update(co_model *m, const unit_buf *ub, int nvalid) {
  for (int j = 0; j < nvalid; j++) {
    int smp[CO_ORDERS];
    for (int o = 0; o < CO_ORDERS; o++) smp[o] = ub->smp[o * ub->unit + j];
    mixer_update(m->w, ub->cxt[j], smp, ub->y[j], ub->pr[j]);
  }
  for (int o = 0; o < CO_ORDERS; o++) {
    uint8_t *st = m->states + (size_t)o * CO_SLOTS;
    for (int j = 0; j < nvalid; j++) sm_update(st, m->statep[o], ub->hash[o * ub->unit + j], ub->y[j]);
  }
}

size_t co_chunk_bound(size_t cs) { return 32 * cs + 1; }

size_t co_encode_chunk(co_model *work, const uint8_t *chunk, size_t len, size_t cs, int unit,
                       uint8_t *out, size_t cap) {
  tables_once();
  unit_buf ub;
  if (unit_buf_init(&ub, unit) != 0) {
    unit_buf_free(&ub);
    return (size_t)-1;
  }
  uint32_t x1 = 0, x2 = 0xffffffffu;
  size_t off = 0;
  uint64_t iters = 8 * (uint64_t)cs / (uint64_t)unit + 1; /* cucm_compress_v2.cu:1067 */
  for (uint64_t u = 0; u < iters; u++) {
    uint64_t base = u * (uint64_t)unit;
    int nvalid = unit_predict(work, chunk, len, cs, base, &ub);
    /* cudaencodeUnit (cucm_compress_v2.cu:841-868): codes prm[0..unit)
     * while inside the chunk, without an input-end check, so the last
     * partial chunk of a stream re-codes stale entries up to 8*cs bits. */
    for (int j = 0; j < unit; j++) {
      if (base + (uint64_t)j >= 8 * (uint64_t)cs) break;
      int pr = ub.prm[j] >> 1, y = ub.prm[j] & 1;
      uint32_t xmid = coder_mid(x1, x2, pr);
      if (y) x2 = xmid; else x1 = xmid + 1;
      while (((x1 ^ x2) & 0xff000000u) == 0) {
        if (off >= cap) {
          unit_buf_free(&ub);
          return (size_t)-1;
        }
        out[off++] = (uint8_t)(x2 >> 24);
        x1 <<= 8;
        x2 = (x2 << 8) | 255u;
      }
    }
    unit_update(work, &ub, nvalid);
  }
  unit_buf_free(&ub);
  if (off >= cap) return (size_t)-1;
  out[off++] = (uint8_t)(x1 >> 24); /* flush byte, cucm_compress_v2.cu:902 */
  return off;
}

void co_decode_chunk(co_model *work, const uint8_t *payload, size_t plen, size_t len, size_t cs,
                     int unit, uint8_t *out) {
  tables_once();
  unit_buf ub;
  if (unit_buf_init(&ub, unit) != 0) {
    unit_buf_free(&ub);
    return;
  }
  memset(out, 0, len);
  uint32_t x1 = 0, x2 = 0xffffffffu, x = 0;
  size_t ioff = 0;
  /* x primes from the first 4 payload bytes (cucm_decompress_v2.cu:967-972);
   * bytes past the payload read as 255 (cucm_decompress_v2.cu:837-843). */
  for (int i = 0; i < 4; i++) x = (x << 8) | (ioff < plen ? payload[ioff++] : 255u);
  uint64_t nbits = 8 * (uint64_t)(len < cs ? len : cs);
  for (uint64_t base = 0; base < nbits; base += (uint64_t)unit) {
    int nvalid = 0;
    for (int j = 0; j < unit && base + (uint64_t)j < nbits; j++) {
      uint64_t b = base + (uint64_t)j;
      size_t byte = (size_t)(b >> 3);
      int bit = (int)(b & 7);
      uint32_t hs[CO_ORDERS];
      bit_hashes(out, byte, bit, hs);
      int smp[CO_ORDERS];
      for (int o = 0; o < CO_ORDERS; o++) {
        uint8_t s = work->states[(size_t)o * CO_SLOTS + hs[o]];
        smp[o] = g_stretch[work->statep[o][s] >> 20];
        ub.hash[o * unit + j] = hs[o];
        ub.smp[o * unit + j] = smp[o];
      }
      int c1 = byte >= 1 ? out[byte - 1] : 0;
      int cxt = mixer_cxt(smp, c1);
      int pr = mixer_pr(work->w, cxt, smp);
      uint32_t xmid = coder_mid(x1, x2, pr);
      int y = x <= xmid;
      if (y) x2 = xmid; else x1 = xmid + 1;
      while (((x1 ^ x2) & 0xff000000u) == 0) {
        x1 <<= 8;
        x2 = (x2 << 8) | 255u;
        x = (x << 8) | (ioff < plen ? payload[ioff++] : 255u);
      }
      out[byte] |= (uint8_t)(y << (7 - bit));
      ub.cxt[j] = cxt;
      ub.pr[j] = pr;
      ub.y[j] = y;
      nvalid++;
    }
    unit_update(work, &ub, nvalid);
  }
  unit_buf_free(&ub);
}

/* ---- fixed-model chunk coder (PDF section 4.5) --------------------------- */

/* The fixed-model variant the paper discusses (section 4.5: the model is
 * kept fixed after the prelearn pass, no online updates): every data bit of
 * the chunk is predicted by the prelearned model exactly as the prelearn
 * pass predicts it (prelearn_bit, i.e. cucm_compress_v2.cu:930-955 --
 * hashes over the chunk's own history, StateMaps, Mixer) and nothing is
 * updated.  The reference ships no code for it; this restatement defines the
 * variant's stream.  Only the chunk's data bits are coded (no stale tail),
 * then the flush byte. */
size_t co_encode_chunk_fixed(const co_model *m, const uint8_t *chunk, size_t len, uint8_t *out, size_t cap) {
  tables_once();
  uint32_t x1 = 0, x2 = 0xffffffffu;
  size_t off = 0;
  uint32_t hs[CO_ORDERS];
  int smp[CO_ORDERS], pr, cxt;
  for (size_t pos = 0; pos < len * 8; pos++) {
    int y = (chunk[pos >> 3] >> (7 - (pos & 7))) & 1;
    prelearn_bit((co_model *)m, chunk, pos, y, &pr, hs, smp, &cxt);
    uint32_t xmid = coder_mid(x1, x2, pr);
    if (y) x2 = xmid; else x1 = xmid + 1;
    while (((x1 ^ x2) & 0xff000000u) == 0) {
      if (off >= cap) return (size_t)-1;
      out[off++] = (uint8_t)(x2 >> 24);
      x1 <<= 8;
      x2 = (x2 << 8) | 255u;
    }
  }
  if (off >= cap) return (size_t)-1;
  out[off++] = (uint8_t)(x1 >> 24);
  return off;
}

void co_decode_chunk_fixed(const co_model *m, const uint8_t *payload, size_t plen, size_t len, uint8_t *out) {
  tables_once();
  memset(out, 0, len);
  uint32_t x1 = 0, x2 = 0xffffffffu, x = 0;
  size_t ioff = 0;
  for (int i = 0; i < 4; i++) x = (x << 8) | (ioff < plen ? payload[ioff++] : 255u);
  uint32_t hs[CO_ORDERS];
  int smp[CO_ORDERS], pr, cxt;
  for (size_t pos = 0; pos < len * 8; pos++) {
    prelearn_bit((co_model *)m, out, pos, 0, &pr, hs, smp, &cxt);
    uint32_t xmid = coder_mid(x1, x2, pr);
    int y = x <= xmid;
    if (y) x2 = xmid; else x1 = xmid + 1;
    while (((x1 ^ x2) & 0xff000000u) == 0) {
      x1 <<= 8;
      x2 = (x2 << 8) | 255u;
      x = (x << 8) | (ioff < plen ? payload[ioff++] : 255u);
    }
    out[pos >> 3] |= (uint8_t)(y << (7 - (pos & 7)));
  }
}

/* ---- container ---------------------------------------------------------- */

static inline void put_be32(uint8_t *p, uint32_t v) {
  p[0] = (uint8_t)(v >> 24);
  p[1] = (uint8_t)(v >> 16);
  p[2] = (uint8_t)(v >> 8);
  p[3] = (uint8_t)v;
}
static inline uint32_t get_be32(const uint8_t *p) {
  return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
}
static inline void put_le32(uint8_t *p, uint32_t v) {
  p[0] = (uint8_t)v;
  p[1] = (uint8_t)(v >> 8);
  p[2] = (uint8_t)(v >> 16);
  p[3] = (uint8_t)(v >> 24);
}
static inline uint32_t get_le32(const uint8_t *p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

typedef struct job {
  const co_model *init;
  const uint8_t *data;  /* whole chunked region */
  size_t n;             /* bytes in the chunked region */
  size_t cs;
  int unit;
  size_t nchunks;
  /* compress */
  uint8_t **pay;
  size_t *pay_n;
  /* decompress */
  const uint8_t *const *cin;
  const size_t *cin_n;
  uint8_t *dout;
  size_t next;          /* next chunk index (shared, under lock) */
  pthread_mutex_t lock;
  int err;
  int decode;
  int fixed;            /* fixed-model variant: the shared model is only read */
} job;

static void *job_worker(void *arg) {
  job *J = (job *)arg;
  co_model *work = J->fixed ? NULL : co_model_new();
  if (!work && !J->fixed) {
    pthread_mutex_lock(&J->lock);
    J->err = -1;
    pthread_mutex_unlock(&J->lock);
    return NULL;
  }
  for (;;) {
    pthread_mutex_lock(&J->lock);
    size_t k = J->next++;
    pthread_mutex_unlock(&J->lock);
    if (k >= J->nchunks) break;
    if (!J->fixed) co_model_copy(work, J->init);
    size_t off = k * J->cs;
    size_t len = J->n - off < J->cs ? J->n - off : J->cs;
    if (!J->decode) {
      size_t cap = co_chunk_bound(J->cs);
      uint8_t *buf = (uint8_t *)malloc(cap);
      size_t got = !buf ? (size_t)-1
                   : J->fixed ? co_encode_chunk_fixed(J->init, J->data + off, len, buf, cap)
                              : co_encode_chunk(work, J->data + off, len, J->cs, J->unit, buf, cap);
      if (got == (size_t)-1) {
        free(buf);
        pthread_mutex_lock(&J->lock);
        J->err = -1;
        pthread_mutex_unlock(&J->lock);
        continue;
      }
      J->pay[k] = buf;
      J->pay_n[k] = got;
    } else if (J->fixed) {
      co_decode_chunk_fixed(J->init, J->cin[k], J->cin_n[k], len, J->dout + off);
    } else {
      co_decode_chunk(work, J->cin[k], J->cin_n[k], len, J->cs, J->unit, J->dout + off);
    }
  }
  if (work) co_model_free(work);
  return NULL;
}

static int run_jobs(job *J, int threads) {
  if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
  if (threads < 1) threads = 1;
  if ((size_t)threads > J->nchunks) threads = (int)(J->nchunks ? J->nchunks : 1);
  pthread_mutex_init(&J->lock, NULL);
  J->next = 0;
  J->err = 0;
  pthread_t *th = (pthread_t *)calloc(threads, sizeof(pthread_t));
  for (int t = 0; t < threads; t++) pthread_create(&th[t], NULL, job_worker, J);
  for (int t = 0; t < threads; t++) pthread_join(th[t], NULL);
  free(th);
  pthread_mutex_destroy(&J->lock);
  return J->err;
}

/* compress_file (cucm_compress_v2.cu:1151-1250); `fixed` selects the
 * fixed-model variant (flag byte bit 1, prelearn required). */
int co_compress_ex(const uint8_t *in, size_t n, size_t cs, int unit, size_t prelearn, int batch, int fixed,
                   int threads, uint8_t **out, size_t *out_n) {
  tables_once();
  if (cs == 0 || unit <= 0 || batch <= 0 || prelearn > n) return -2;
  if (fixed && prelearn == 0) return -2;
  co_model *init = co_model_new();
  if (!init) return -1;
  size_t pl_cap = prelearn * 8 + 8;
  uint8_t *pl = (uint8_t *)malloc(pl_cap);
  size_t pl_coded = 0;
  if (prelearn > 0) pl_coded = co_prelearn_encode(init, in, prelearn, pl, pl_cap);
  int raw = prelearn <= pl_coded; /* cucm_compress_v2.cu:1217-1223 */
  size_t pl_len = raw ? prelearn : pl_coded;

  size_t body_n = n - prelearn;
  size_t nchunks = (body_n + cs - 1) / cs;
  job J;
  memset(&J, 0, sizeof J);
  J.init = init;
  J.data = in + prelearn;
  J.n = body_n;
  J.cs = cs;
  J.unit = unit;
  J.nchunks = nchunks;
  J.fixed = fixed;
  J.pay = (uint8_t **)calloc(nchunks ? nchunks : 1, sizeof(uint8_t *));
  J.pay_n = (size_t *)calloc(nchunks ? nchunks : 1, sizeof(size_t));
  int rc = nchunks ? run_jobs(&J, threads) : 0;
  co_model_free(init);
  if (rc != 0) {
    for (size_t k = 0; k < nchunks; k++) free(J.pay[k]);
    free(J.pay);
    free(J.pay_n);
    free(pl);
    return rc;
  }
  size_t nbatches = (nchunks + (size_t)batch - 1) / (size_t)batch;
  size_t total = 21 + pl_len + 4 * nbatches + 4 * nchunks;
  for (size_t k = 0; k < nchunks; k++) total += J.pay_n[k];
  uint8_t *o = (uint8_t *)malloc(total);
  /* header, cucm_compress_v2.cu:1197-1216 (all fields big-endian) */
  put_be32(o, (uint32_t)n);
  o[4] = (uint8_t)(batch >> 8);
  o[5] = (uint8_t)batch;
  o[6] = (uint8_t)(unit >> 8);
  o[7] = (uint8_t)unit;
  put_be32(o + 8, (uint32_t)cs);
  put_be32(o + 12, (uint32_t)pl_coded);
  put_be32(o + 16, (uint32_t)prelearn);
  o[20] = (uint8_t)((raw ? 0 : 1) | (fixed ? 2 : 0));
  memcpy(o + 21, raw ? in : pl, pl_len);
  size_t w = 21 + pl_len;
  for (size_t b = 0; b < nbatches; b++) {
    size_t k0 = b * (size_t)batch;
    size_t k1 = k0 + (size_t)batch < nchunks ? k0 + (size_t)batch : nchunks;
    size_t c = k1 - k0;
    size_t bsz = 4 * c;
    for (size_t k = k0; k < k1; k++) bsz += J.pay_n[k];
    put_le32(o + w, (uint32_t)bsz); /* host-order u32, cucm_compress_v2.cu:1241-1243 */
    w += 4;
    /* end offsets (cudaencodefinal, cucm_compress_v2.cu:903-907):
     * index of each chunk's last byte, counted from the batch body start */
    size_t acc = 4 * c - 1;
    for (size_t k = k0; k < k1; k++) {
      acc += J.pay_n[k];
      put_be32(o + w + 4 * (k - k0), (uint32_t)acc);
    }
    w += 4 * c;
    for (size_t k = k0; k < k1; k++) {
      memcpy(o + w, J.pay[k], J.pay_n[k]);
      w += J.pay_n[k];
      free(J.pay[k]);
    }
  }
  free(J.pay);
  free(J.pay_n);
  free(pl);
  *out = o;
  *out_n = w;
  return 0;
}

int co_compress(const uint8_t *in, size_t n, size_t cs, int unit, size_t prelearn, int batch, int threads,
                uint8_t **out, size_t *out_n) {
  return co_compress_ex(in, n, cs, unit, prelearn, batch, 0, threads, out, out_n);
}

/* decompress (cucm_decompress_v2.cu:1185-1248); flag bit 1 is the
 * fixed-model variant. */
int co_decompress(const uint8_t *in, size_t n, int threads, uint8_t **out, size_t *out_n) {
  tables_once();
  if (n < 21) return -3;
  size_t total = get_be32(in);
  int batch = (in[4] << 8) | in[5];
  int unit = (in[6] << 8) | in[7];
  size_t cs = get_be32(in + 8);
  size_t pl_coded = get_be32(in + 12);
  size_t prelearn = get_be32(in + 16);
  int coded = in[20] & 1;
  int fixed = (in[20] & 2) != 0;
  if (cs == 0 || unit <= 0 || batch <= 0 || prelearn > total || (fixed && !prelearn)) return -3;
  size_t pl_len = coded ? pl_coded : prelearn;
  if (21 + pl_len > n) return -3;
  uint8_t *o = (uint8_t *)calloc(total ? total : 1, 1);
  co_model *init = co_model_new();
  if (!o || !init) {
    free(o);
    co_model_free(init);
    return -1;
  }
  if (prelearn) {
    if (coded) co_prelearn_decode(init, in + 21, pl_len, o, prelearn);
    else {
      memcpy(o, in + 21, prelearn);
      co_prelearn_train(init, o, prelearn);
    }
  }
  size_t r = 21 + pl_len;
  size_t body_n = total - prelearn;
  size_t nchunks = (body_n + cs - 1) / cs;
  size_t nbatches = (nchunks + (size_t)batch - 1) / (size_t)batch;
  const uint8_t **cin = (const uint8_t **)calloc(nchunks ? nchunks : 1, sizeof(uint8_t *));
  size_t *cin_n = (size_t *)calloc(nchunks ? nchunks : 1, sizeof(size_t));
  int rc = 0;
  for (size_t b = 0; b < nbatches && rc == 0; b++) {
    size_t k0 = b * (size_t)batch;
    size_t k1 = k0 + (size_t)batch < nchunks ? k0 + (size_t)batch : nchunks;
    size_t c = k1 - k0;
    if (r + 4 + 4 * c > n) { rc = -3; break; }
    size_t bsz = get_le32(in + r);
    r += 4;
    if (bsz < 4 * c || r + bsz > n) { rc = -3; break; }
    const uint8_t *body = in + r + 4 * c;
    size_t body_len = bsz - 4 * c;
    size_t start = 0;
    for (size_t k = k0; k < k1; k++) {
      /* chunkstarts[i+1] = end_i - 4C + 1 (cucm_decompress_v2.cu:1231-1237) */
      size_t end = (size_t)get_be32(in + r + 4 * (k - k0)) + 1 - 4 * c;
      if (end < start || end > body_len) { rc = -3; break; }
      cin[k] = body + start;
      cin_n[k] = end - start;
      start = end;
    }
    r += bsz;
  }
  if (rc == 0 && nchunks) {
    job J;
    memset(&J, 0, sizeof J);
    J.init = init;
    J.n = body_n;
    J.cs = cs;
    J.unit = unit;
    J.nchunks = nchunks;
    J.cin = cin;
    J.cin_n = cin_n;
    J.dout = o + prelearn;
    J.decode = 1;
    J.fixed = fixed;
    rc = run_jobs(&J, threads);
  }
  free(cin);
  free(cin_n);
  co_model_free(init);
  if (rc != 0) {
    free(o);
    return rc;
  }
  *out = o;
  *out_n = total;
  return 0;
}
