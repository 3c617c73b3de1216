// container.cuh -- the reference's container format on the host, and the
// pack kernel that lays chunk payloads out as batches.
//
// compress_file (cucm_compress_v2.cu:1151-1250) writes a 21-byte big-endian
// header, the prelearn block, then per batch of up to -b chunks a host-order
// (little-endian) u32 size, C big-endian u32 chunk end offsets and the chunk
// payloads; decompress (cucm_decompress_v2.cu:1185-1248) reads it back.
// Shared by the context API (api.cu) and the serving loop (serve.cu); each
// includes it inside an anonymous namespace.
#pragma once

constexpr uint64_t kHeaderBytes = 21;

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
  uint32_t end_value;  // big-endian field value
  uint32_t batch_size; // valid when size_at != ~0
  uint64_t size_at;    // body offset of the batch size field or ~0
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
    uint8_t *t = p.base + p.table_at;
    t[0] = (uint8_t)(p.end_value >> 24);
    t[1] = (uint8_t)(p.end_value >> 16);
    t[2] = (uint8_t)(p.end_value >> 8);
    t[3] = (uint8_t)p.end_value;
    if (p.size_at != ~0ull) {
      uint8_t *z = p.base + p.size_at;
      z[0] = (uint8_t)p.batch_size;
      z[1] = (uint8_t)(p.batch_size >> 8);
      z[2] = (uint8_t)(p.batch_size >> 16);
      z[3] = (uint8_t)(p.batch_size >> 24);
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
  if (n > 0xffffffffull) return CUCM_EINVAL;  // header field is 32 bits
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
  hdr.assign(kHeaderBytes + pl_len, 0);
  put_be32(&hdr[0], (uint32_t)n);
  hdr[4] = (uint8_t)(p->batch >> 8);
  hdr[5] = (uint8_t)p->batch;
  hdr[6] = (uint8_t)(p->unit >> 8);
  hdr[7] = (uint8_t)p->unit;
  put_be32(&hdr[8], (uint32_t)p->chunksize);
  put_be32(&hdr[12], (uint32_t)coded);
  put_be32(&hdr[16], (uint32_t)p->prelearn);
  hdr[20] = raw ? 0 : 1;
  if (pl_len) std::memcpy(&hdr[kHeaderBytes], raw ? in : pl.data(), pl_len);
  return CUCM_OK;
}

struct Parsed {
  uint64_t total, cs, prelearn, pl_coded, pl_len;
  uint32_t batch, unit;
  int coded;
};

inline int parse_header(const uint8_t *in, uint64_t n, Parsed &h) {
  if (!in || n < kHeaderBytes) return CUCM_EFORMAT;
  h.total = get_be32(in);
  h.batch = ((uint32_t)in[4] << 8) | in[5];
  h.unit = ((uint32_t)in[6] << 8) | in[7];
  h.cs = get_be32(in + 8);
  h.pl_coded = get_be32(in + 12);
  h.prelearn = get_be32(in + 16);
  h.coded = in[20];
  if (h.cs == 0 || h.batch == 0 || h.unit < 32 || h.unit > (uint32_t)kMaxUnit || h.unit % 32) return CUCM_EFORMAT;
  if (h.prelearn > h.total) return CUCM_EFORMAT;
  h.pl_len = h.coded ? h.pl_coded : h.prelearn;
  if (kHeaderBytes + h.pl_len > n) return CUCM_EFORMAT;
  return CUCM_OK;
}

// Chunk payload extents of the batches that follow the prelearn block
// (cucm_decompress_v2.cu:1223-1237).  Offsets are relative to `body`.
inline int parse_batches(const uint8_t *body, uint64_t body_n, uint64_t nchunks, uint32_t batch, bool with_sizes,
                  std::vector<uint64_t> &off, std::vector<uint64_t> &len) {
  off.resize(nchunks);
  len.resize(nchunks);
  uint64_t r = 0;
  const uint64_t nb = (nchunks + batch - 1) / batch;
  for (uint64_t b = 0; b < nb; b++) {
    uint64_t k0 = b * batch, k1 = std::min<uint64_t>(k0 + batch, nchunks), C = k1 - k0;
    uint64_t bsz;
    if (with_sizes) {
      if (r + 4 > body_n) return CUCM_EFORMAT;
      bsz = get_le32(body + r);
      r += 4;
    } else {
      bsz = body_n - r;
    }
    if (bsz < 4 * C || r + bsz > body_n) return CUCM_EFORMAT;
    const uint64_t pay0 = r + 4 * C;
    const uint64_t pay_n = bsz - 4 * C;
    uint64_t start = 0;
    for (uint64_t k = k0; k < k1; k++) {
      uint64_t endv = get_be32(body + r + 4 * (k - k0));
      if (endv + 1 < 4 * C) return CUCM_EFORMAT;
      uint64_t end = endv + 1 - 4 * C;
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
inline uint64_t layout_chunks(const uint64_t *lens, const uint8_t *const *src, uint64_t nchunks, uint32_t batch,
                              bool with_sizes, uint8_t *base, std::vector<PackEntry> *pe) {
  const uint64_t nb = (nchunks + batch - 1) / batch;
  uint64_t w = 0;
  for (uint64_t b = 0; b < nb; b++) {
    const uint64_t k0 = b * batch, k1 = std::min<uint64_t>(k0 + batch, nchunks), C = k1 - k0;
    uint64_t bsz = 4 * C;
    for (uint64_t k = k0; k < k1; k++) bsz += lens[k];
    const uint64_t size_at = w;
    if (with_sizes) w += 4;
    const uint64_t table = w;
    w += 4 * C;
    uint64_t acc = 4 * C - 1;
    for (uint64_t k = k0; k < k1; k++) {
      acc += lens[k];
      if (pe) {
        PackEntry p;
        p.src = src[k];
        p.base = base;
        p.dst = w;
        p.len = lens[k];
        p.table_at = table + 4 * (k - k0);
        p.end_value = (uint32_t)acc;
        p.size_at = (k == k0 && with_sizes) ? size_at : ~0ull;
        p.batch_size = (uint32_t)bsz;
        pe->push_back(p);
      }
      w += lens[k];
    }
  }
  return w;
}

