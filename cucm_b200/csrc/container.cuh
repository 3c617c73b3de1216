// container.cuh -- the reference's container format on the host, and the
// pack kernel that lays chunk payloads out as batches.
//
// compress_file (cucm_compress_v2.cu:1151-1250) writes a 21-byte big-endian
// header, the prelearn block, then per batch of up to -b chunks a host-order
// (little-endian) u32 size, C big-endian u32 chunk end offsets and the chunk
// payloads; decompress (cucm_decompress_v2.cu:1185-1248) reads it back.
// Shared by the context API (api.cu) and the serving loop (serve.cu); each
// includes it inside an anonymous namespace.
//
// Those 32-bit fields cap a reference container at 4 GiB of input (and the
// reference truncates a batch size past 4 GiB without a word,
// cucm_compress_v2.cu:1241).  Larger streams get the 64-bit container, a
// format of this library only: bytes 0..3 are 0xffffffff and bytes 4..5 zero
// (a batch count of 0, which no reference container has, so a 32-bit reader
// refuses it), bytes 6..7 the version 2; then, big-endian, the original size
// (u64), batch (u32), unit (u32), chunk size (u32), prelearn coded size
// (u64), prelearn raw size (u64) and the flag byte -- 45 bytes -- and per
// batch a little-endian u64 size and big-endian u64 chunk end offsets.  The
// chunk payloads are the same bytes in both formats.
#pragma once

constexpr uint64_t kHeaderBytes = 21;    // the reference's header
constexpr uint64_t kHeaderBytes64 = 45;  // the 64-bit container's header

// ---------------------------------------------------------------------------
// Pack kernel: one CTA per chunk copies its payload from scratch into the
// container, writes its big-endian end offset, and the first chunk of a batch
// writes the batch's little-endian size field.
struct PackEntry {
  const uint8_t *src;  // payload in scratch
  uint8_t *base;       // start of the container body it goes to
  uint64_t dst;        // body offset of the payload
  uint64_t len;        // payload bytes
  uint64_t table_at;   // body offset of this chunk's end-offset field
  uint64_t end_value;  // big-endian field value
  uint64_t batch_size; // valid when size_at != ~0
  uint64_t size_at;    // body offset of the batch size field or ~0
  uint32_t wide;       // 8-byte fields (64-bit container) instead of 4
};

// One CTA per chunk: payload copy plus its end-offset field (and the batch
// size field for the first chunk of a batch), cudaencodefinal's packing
// (cucm_compress_v2.cu:880-914).
__global__ void pack_kernel(const PackEntry *e, uint32_t n) {
  const uint32_t k = blockIdx.x;
  if (k >= n) return;
  const PackEntry p = e[k];
  const uint8_t *s = p.src;
  uint8_t *d = p.base + p.dst;
  for (uint64_t i = threadIdx.x; i < p.len; i += blockDim.x) d[i] = s[i];
  if (threadIdx.x == 0) {
    const int w = p.wide ? 8 : 4;
    uint8_t *t = p.base + p.table_at;
    for (int b = 0; b < w; b++) t[b] = (uint8_t)(p.end_value >> (8 * (w - 1 - b)));
    if (p.size_at != ~0ull) {
      uint8_t *z = p.base + p.size_at;
      for (int b = 0; b < w; b++) z[b] = (uint8_t)(p.batch_size >> (8 * b));
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
inline void put_be64(uint8_t *p, uint64_t v) {
  for (int b = 0; b < 8; b++) p[b] = (uint8_t)(v >> (8 * (7 - b)));
}
inline uint64_t get_be64(const uint8_t *p) {
  uint64_t v = 0;
  for (int b = 0; b < 8; b++) v = (v << 8) | p[b];
  return v;
}
inline uint64_t get_le64(const uint8_t *p) {
  uint64_t v = 0;
  for (int b = 7; b >= 0; b--) v = (v << 8) | p[b];
  return v;
}
// Big-endian end offset / little-endian batch size, 4 or 8 bytes.
inline uint64_t get_be(const uint8_t *p, bool wide) { return wide ? get_be64(p) : get_be32(p); }
inline uint64_t get_le(const uint8_t *p, bool wide) { return wide ? get_le64(p) : get_le32(p); }

// The container a stream is written in: the reference's 32-bit one unless
// the caller asks for the 64-bit one or the input needs it.
inline bool wide_format(const cucm_params *p, uint64_t n) {
  return p->format == CUCM_FORMAT_64 || (p->format == CUCM_FORMAT_AUTO && n > 0xffffffffull);
}

inline uint64_t scratch_cap(uint64_t cs) {
  // Typical payloads stay below ~1.1x the chunk; 2x + 4 KiB leaves margin.
  // A chunk that still overflows is re-coded with the hard bound.
  uint64_t c = 2 * cs + 4096;
  uint64_t hard = 32 * cs + 16;
  return ((c < hard ? c : hard) + 15) & ~15ull;
}
inline uint64_t hard_cap(uint64_t cs) { return (32 * cs + 1 + 15) & ~15ull; }

// Validate stream parameters the way the reference's container can hold them.
inline int check_params(const cucm_params *p, uint64_t n) {
  if (!p) return CUCM_EINVAL;
  if (p->chunksize == 0 || p->chunksize > 0xffffffffull) return CUCM_EINVAL;
  if (p->unit < 32 || p->unit > (uint32_t)kMaxUnit || p->unit % 32) return CUCM_EINVAL;
  if (p->batch == 0 || p->batch > 0xffff) return CUCM_EINVAL;
  if (p->prelearn > n) return CUCM_EINVAL;
  if (p->format != CUCM_FORMAT_AUTO && p->format != CUCM_FORMAT_32 && p->format != CUCM_FORMAT_64) return CUCM_EINVAL;
  if (p->fixed_model > 1 || (p->fixed_model && p->prelearn == 0)) return CUCM_EINVAL;  // the variant needs a prelearned model
  if (!wide_format(p, n) && n > 0xffffffffull) return CUCM_EINVAL;  // the 32-bit header holds the size
  return CUCM_OK;
}

// Container header + prelearn block.  Also produces the initial model.
inline int make_header(const uint8_t *in, uint64_t n, const cucm_params *p, std::vector<uint8_t> &hdr,
                std::unique_ptr<HostModel> &hm) {
  std::vector<uint8_t> pl;
  uint64_t coded = 0;
  if (p->prelearn > 0) {
    hm.reset(new HostModel());
    coded = hm->prelearn_encode(in, p->prelearn, pl);
  }
  const bool raw = p->prelearn <= coded;  // cucm_compress_v2.cu:1217-1223
  const uint64_t pl_len = raw ? p->prelearn : coded;
  const bool wide = wide_format(p, n);
  const uint64_t hl = wide ? kHeaderBytes64 : kHeaderBytes;
  hdr.assign(hl + pl_len, 0);
  if (!wide) {
    put_be32(&hdr[0], (uint32_t)n);
    hdr[4] = (uint8_t)(p->batch >> 8);
    hdr[5] = (uint8_t)p->batch;
    hdr[6] = (uint8_t)(p->unit >> 8);
    hdr[7] = (uint8_t)p->unit;
    put_be32(&hdr[8], (uint32_t)p->chunksize);
    put_be32(&hdr[12], (uint32_t)coded);
    put_be32(&hdr[16], (uint32_t)p->prelearn);
    hdr[20] = (uint8_t)((raw ? 0 : 1) | (p->fixed_model ? 2 : 0));
  } else {
    put_be32(&hdr[0], 0xffffffffu);  // bytes 4..5 stay zero
    hdr[7] = 2;
    put_be64(&hdr[8], n);
    put_be32(&hdr[16], p->batch);
    put_be32(&hdr[20], p->unit);
    put_be32(&hdr[24], (uint32_t)p->chunksize);
    put_be64(&hdr[28], coded);
    put_be64(&hdr[36], p->prelearn);
    hdr[44] = (uint8_t)((raw ? 0 : 1) | (p->fixed_model ? 2 : 0));
  }
  if (pl_len) std::memcpy(&hdr[hl], raw ? in : pl.data(), pl_len);
  return CUCM_OK;
}

struct Parsed {
  uint64_t total, cs, prelearn, pl_coded, pl_len;
  uint32_t batch, unit;
  int coded;
  int flag;      // flag byte: bit 0 coded prelearn block, bit 1 fixed model
  bool fixed;    // the fixed-model variant
  bool wide;     // the 64-bit container
  uint64_t hdr;  // header bytes (21 or 45); the prelearn block follows
  uint64_t body_off() const { return hdr + pl_len; }
};

// True when the first 8 header bytes mark the 64-bit container.
inline bool is_wide_header(const uint8_t *in, uint64_t n) {
  return n >= 8 && get_be32(in) == 0xffffffffu && in[4] == 0 && in[5] == 0 && in[6] == 0 && in[7] == 2;
}

inline int parse_header(const uint8_t *in, uint64_t n, Parsed &h) {
  if (!in || n < kHeaderBytes) return CUCM_EFORMAT;
  h.wide = is_wide_header(in, n);
  if (!h.wide) {
    h.hdr = kHeaderBytes;
    h.total = get_be32(in);
    h.batch = ((uint32_t)in[4] << 8) | in[5];
    h.unit = ((uint32_t)in[6] << 8) | in[7];
    h.cs = get_be32(in + 8);
    h.pl_coded = get_be32(in + 12);
    h.prelearn = get_be32(in + 16);
    h.flag = in[20];
  } else {
    if (n < kHeaderBytes64) return CUCM_EFORMAT;
    h.hdr = kHeaderBytes64;
    h.total = get_be64(in + 8);
    h.batch = get_be32(in + 16);
    h.unit = get_be32(in + 20);
    h.cs = get_be32(in + 24);
    h.pl_coded = get_be64(in + 28);
    h.prelearn = get_be64(in + 36);
    h.flag = in[44];
  }
  if (h.cs == 0 || h.batch == 0 || h.unit < 32 || h.unit > (uint32_t)kMaxUnit || h.unit % 32) return CUCM_EFORMAT;
  if (h.prelearn > h.total) return CUCM_EFORMAT;
  // flag bit 0: the prelearn block is coded; bit 1: the fixed-model variant
  // (which needs the prelearned model)
  if (h.flag > 3 || ((h.flag & 2) && h.prelearn == 0)) return CUCM_EFORMAT;
  h.coded = h.flag & 1;
  h.fixed = (h.flag & 2) != 0;
  h.pl_len = h.coded ? h.pl_coded : h.prelearn;
  if (h.pl_len > n || h.hdr + h.pl_len > n) return CUCM_EFORMAT;
  return CUCM_OK;
}

// Chunk payload extents of the batches that follow the prelearn block
// (cucm_decompress_v2.cu:1223-1237).  Offsets are relative to `body`.
inline int parse_batches(const uint8_t *body, uint64_t body_n, uint64_t nchunks, uint32_t batch, bool with_sizes,
                         std::vector<uint64_t> &off, std::vector<uint64_t> &len, bool wide = false) {
  off.resize(nchunks);
  len.resize(nchunks);
  const uint64_t w = wide ? 8 : 4;
  uint64_t r = 0;
  const uint64_t nb = (nchunks + batch - 1) / batch;
  for (uint64_t b = 0; b < nb; b++) {
    uint64_t k0 = b * batch, k1 = std::min<uint64_t>(k0 + batch, nchunks), C = k1 - k0;
    uint64_t bsz;
    if (with_sizes) {
      if (r + w > body_n) return CUCM_EFORMAT;
      bsz = get_le(body + r, wide);
      r += w;
    } else {
      bsz = body_n - r;
    }
    if (bsz < w * C || bsz > body_n - r) return CUCM_EFORMAT;
    const uint64_t pay0 = r + w * C;
    const uint64_t pay_n = bsz - w * C;
    uint64_t start = 0;
    for (uint64_t k = k0; k < k1; k++) {
      uint64_t endv = get_be(body + r + w * (k - k0), wide);
      if (endv + 1 < w * C) return CUCM_EFORMAT;
      uint64_t end = endv + 1 - w * C;
      if (end < start || end > pay_n) return CUCM_EFORMAT;
      off[k] = pay0 + start;
      len[k] = end - start;
      start = end;
    }
    r += bsz;
  }
  return CUCM_OK;
}

// Batch layout of n chunks (cudaencodefinal,
// cucm_compress_v2.cu:880-914): per batch an optional u32 little-endian size,
// C big-endian end offsets (offset_i = 4C - 1 + sum of lengths), payloads.
// Appends the pack entries for a body starting at `base` (may be null when
// only the size is wanted) and returns the body size.
// In the 32-bit format a batch size or end offset that does not fit its field
// sets *overflow (the reference would truncate it).
inline uint64_t layout_chunks(const uint64_t *lens, const uint8_t *const *src, uint64_t nchunks, uint32_t batch,
                              bool with_sizes, uint8_t *base, std::vector<PackEntry> *pe, bool wide = false,
                              bool *overflow = nullptr) {
  const uint64_t nb = (nchunks + batch - 1) / batch;
  const uint64_t fw = wide ? 8 : 4;
  uint64_t w = 0;
  for (uint64_t b = 0; b < nb; b++) {
    const uint64_t k0 = b * batch, k1 = std::min<uint64_t>(k0 + batch, nchunks), C = k1 - k0;
    uint64_t bsz = fw * C;
    for (uint64_t k = k0; k < k1; k++) bsz += lens[k];
    if (!wide && bsz > 0xffffffffull && overflow) *overflow = true;
    const uint64_t size_at = w;
    if (with_sizes) w += fw;
    const uint64_t table = w;
    w += fw * C;
    uint64_t acc = fw * C - 1;
    for (uint64_t k = k0; k < k1; k++) {
      acc += lens[k];
      if (pe) {
        PackEntry p;
        p.src = src[k];
        p.base = base;
        p.dst = w;
        p.len = lens[k];
        p.table_at = table + fw * (k - k0);
        p.end_value = acc;
        p.size_at = (k == k0 && with_sizes) ? size_at : ~0ull;
        p.batch_size = bsz;
        p.wide = wide ? 1u : 0u;
        pe->push_back(p);
      }
      w += lens[k];
    }
  }
  return w;
}

