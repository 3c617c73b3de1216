// host_model.h -- the bit-serial host model used by the optional prelearn
// prefix (-p).
//
// In the reference the prelearn pass is host code by design
// (prelearn, cucm_compress_v2.cu:924-981; replay on decode
// cucm_decompress_v2.cu:1056-1182): the first `prelearn` bytes train one
// model bit by bit (update after every bit, no unit freezing) and are coded
// with it; that trained model then initialises every chunk.  This header
// keeps that pass on the host and converts its result into the device slot
// layout (orders 0 and 1 by context, orders 2..7 by 25-bit slot).
#pragma once

#include <cstdint>
#include <cstring>
#include <vector>

#include "engine.cuh"
#include "model.cuh"
#include "tables.h"

namespace cucm {

struct HostModel {
  std::vector<uint8_t> states;  // kOrders << 25
  uint32_t statep[kOrders][256];
  int32_t w[kMixCtx * kOrders];
  Tables t;

  HostModel() : states((size_t)kOrders * kSlots, 0) {
    build_tables(t);
    for (int o = 0; o < kOrders; o++)
      for (int s = 0; s < 256; s++) statep[o][s] = 1u << 31;
    std::memset(w, 0, sizeof w);
  }

  // FNV-1 slot of every order for the bit at `pos` of `buf` (history of the
  // buffer only, zero before its start).
  static void slots(const uint8_t *buf, uint64_t pos, uint32_t out[kOrders]) {
    uint64_t q = pos >> 3;
    int r = (int)(pos & 7);
    uint32_t h0 = (1u << r) | ((uint32_t)buf[q] >> (8 - r));
    uint32_t acc = (kFnvBasis ^ h0) * kFnvPrime;
    out[0] = acc & (kSlots - 1);
    for (int o = 1; o < kOrders; o++) {
      uint32_t prev = q >= (uint64_t)o ? buf[q - o] : 0u;
      acc = (acc ^ prev) * kFnvPrime;
      out[o] = acc & (kSlots - 1);
    }
  }

  int predict(const uint8_t *buf, uint64_t pos, uint32_t sl[kOrders], int smp[kOrders], int *cxt) const {
    slots(buf, pos, sl);
    int olen = 0;
    for (int o = 0; o < kOrders; o++) {
      uint8_t s = states[(size_t)o * kSlots + sl[o]];
      smp[o] = t.stretch[statep[o][s] >> 20];
      olen += smp[o] != 1;
    }
    uint64_t q = pos >> 3;
    int c1 = q >= 1 ? buf[q - 1] : 0;
    int cx = olen + (c1 >> 5) * 10;
    long long sum = 0;
    for (int o = 0; o < kOrders; o++) sum += (long long)w[cx * kOrders + o] * smp[o];
    sum >>= 16;
    int idx = sum < -2047 ? -2047 : (sum > 2048 ? 2048 : (int)sum);
    int pr = t.squash[idx + 2047];
    *cxt = cx;
    return pr < 2048 ? pr + 1 : pr;
  }

  void update(const uint32_t sl[kOrders], const int smp[kOrders], int cx, int y, int pr) {
    int err = ((y << 12) - pr) * 7;
    for (int o = 0; o < kOrders; o++)
      w[cx * kOrders + o] = (int32_t)((uint32_t)w[cx * kOrders + o] +
                                      (uint32_t)(int32_t)(((long long)err * smp[o]) >> 16));
    for (int o = 0; o < kOrders; o++) {
      uint8_t &st = states[(size_t)o * kSlots + sl[o]];
      uint32_t &v = statep[o][st];
      v = statep_next(v, y, t.dt[v & 1023u]);
      st = t.nex[st][y];
    }
  }

  // Code `n` bytes, training as we go.  Returns the coded size.
  size_t prelearn_encode(const uint8_t *in, size_t n, std::vector<uint8_t> &out) {
    out.clear();
    uint32_t x1 = 0, x2 = 0xffffffffu;
    uint32_t sl[kOrders];
    int smp[kOrders], cx;
    for (uint64_t pos = 0; pos < 8ull * n; pos++) {
      int y = (in[pos >> 3] >> (7 - (pos & 7))) & 1;
      int pr = predict(in, pos, sl, smp, &cx);
      update(sl, smp, cx, y, pr);
      uint32_t xmid = coder_mid(x1, x2, (uint32_t)pr);
      if (y) x2 = xmid; else x1 = xmid + 1;
      while (((x1 ^ x2) & 0xff000000u) == 0) {
        out.push_back((uint8_t)(x2 >> 24));
        x1 <<= 8;
        x2 = (x2 << 8) | 255u;
      }
    }
    out.push_back((uint8_t)(x1 >> 24));
    return out.size();
  }

  void prelearn_train(const uint8_t *in, size_t n) {
    uint32_t sl[kOrders];
    int smp[kOrders], cx;
    for (uint64_t pos = 0; pos < 8ull * n; pos++) {
      int y = (in[pos >> 3] >> (7 - (pos & 7))) & 1;
      int pr = predict(in, pos, sl, smp, &cx);
      update(sl, smp, cx, y, pr);
    }
  }

  void prelearn_decode(const uint8_t *in, size_t in_n, uint8_t *out, size_t n) {
    std::memset(out, 0, n);
    uint32_t x1 = 0, x2 = 0xffffffffu, x = 0;
    size_t ioff = 0;
    for (int i = 0; i < 4; i++) x = (x << 8) | (ioff < in_n ? in[ioff++] : 255u);
    uint32_t sl[kOrders];
    int smp[kOrders], cx;
    for (uint64_t pos = 0; pos < 8ull * n; pos++) {
      int pr = predict(out, pos, sl, smp, &cx);
      uint32_t xmid = coder_mid(x1, x2, (uint32_t)pr);
      int y = x <= xmid;
      if (y) x2 = xmid; else x1 = xmid + 1;
      update(sl, smp, cx, y, pr);
      while (((x1 ^ x2) & 0xff000000u) == 0) {
        x1 <<= 8;
        x2 = (x2 << 8) | 255u;
        x = (x << 8) | (ioff < in_n ? in[ioff++] : 255u);
      }
      out[pos >> 3] |= (uint8_t)(y << (7 - (pos & 7)));
    }
  }

  // Device layout: slot image (kSlotTableBytes) and statep/weights.
  void to_device(std::vector<uint8_t> &image, ModelInit &mi) const {
    image.assign(kSlotTableBytes, 0);
    for (uint32_t h0 = 1; h0 < 256; h0++) {
      uint32_t acc = (kFnvBasis ^ h0) * kFnvPrime;
      image[h0] = states[acc & (kSlots - 1)];
      for (uint32_t c1 = 0; c1 < 256; c1++) {
        uint32_t a1 = (acc ^ c1) * kFnvPrime;
        image[kOrder1Off + ((c1 << 8) | h0)] = states[(size_t)kSlots + (a1 & (kSlots - 1))];
      }
    }
    std::memcpy(image.data() + kHashedOff, states.data() + 2ull * kSlots, 6ull * kSlots);
    std::memcpy(mi.statep, statep, sizeof statep);
    std::memcpy(mi.w, w, sizeof w);
  }
};

}  // namespace cucm
