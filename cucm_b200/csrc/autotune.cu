// autotune.cu -- measured choice of the execution form (cucm_autotune).
//
// The reference fixes its launch shapes; here the launch form, the
// compressor's CTAs per SM, the warps per chunk (the pipelined kernels: 7
// warps per chunk to compress, a pair to decode; the generic kernels: 8
// warps per chunk), the decoder's chunks per CTA and its order 0/1 table
// placement are execution choices that never change an output byte.  The autotuner runs every candidate
// through the public entry points on the caller's sample, checks that all of
// them give the same container and give the sample back, and applies the
// one with the least compress + decompress device time.
#include <cstdint>
#include <cstring>
#include <vector>

#include "cucm.h"

namespace {

// Fastest of `reps` compressions; `out` receives the container.
int timed_compress(cucm_ctx *c, const uint8_t *in, uint64_t n, const cucm_params *p, int reps,
                   std::vector<uint8_t> &out, double &best_ms) {
  const uint64_t cap = cucm_compress_bound(n, p);
  out.assign(cap ? cap : 1, 0);
  best_ms = -1.0;
  uint64_t got = 0;
  for (int r = 0; r < reps; r++) {
    const int rc = cucm_compress(c, in, n, p, out.data(), cap, &got);
    if (rc) return rc;
    cucm_stats st;
    cucm_last_stats(c, &st);
    if (best_ms < 0.0 || st.device_ms < best_ms) best_ms = st.device_ms;
  }
  out.resize(got);
  return CUCM_OK;
}

// Fastest of `reps` decompressions, each checked against the sample.
int timed_decompress(cucm_ctx *c, const std::vector<uint8_t> &comp, const uint8_t *want, uint64_t n, int reps,
                     std::vector<uint8_t> &back, double &best_ms) {
  back.assign(n, 0);
  best_ms = -1.0;
  for (int r = 0; r < reps; r++) {
    uint64_t got = 0;
    const int rc = cucm_decompress(c, comp.data(), comp.size(), back.data(), n, &got);
    if (rc) return rc;
    if (got != n || std::memcmp(back.data(), want, n) != 0) return CUCM_EMISMATCH;
    cucm_stats st;
    cucm_last_stats(c, &st);
    if (best_ms < 0.0 || st.device_ms < best_ms) best_ms = st.device_ms;
  }
  return CUCM_OK;
}

}  // namespace

extern "C" int cucm_autotune(cucm_ctx *c, const uint8_t *sample, uint64_t n, const cucm_params *p, int reps,
                             cucm_tune_result *results, uint32_t cap, uint32_t *count, cucm_tuning *best) {
  if (!c || !sample || n == 0 || !p || !best || reps < 1 || (!results && cap)) return CUCM_EINVAL;
  if (count) *count = 0;
  cucm_tuning base;
  int rc = cucm_ctx_get_tuning(c, &base);
  if (rc) return rc;
  auto fail = [&](int code) {
    cucm_ctx_set_tuning(c, &base);
    return code;
  };
  auto candidate = [&](int form) {
    cucm_tune_result r;
    r.tuning = base;
    r.tuning.form = form;
    r.tuning.kernel = 0;
    r.tuning.dec_pairs = 0;
    r.tuning.dec_tables = 0;
    r.tuning.cmp_ctas = 0;
    r.compress_ms = -1.0;
    r.decompress_ms = -1.0;
    return r;
  };

  const int forms[2] = {CUCM_FORM_PERSISTENT, CUCM_FORM_PLAIN};
  std::vector<cucm_tune_result> cands;
  std::vector<uint8_t> ref, out, back;
  {
    // untimed warm-up: the context's first calls allocate its slot tables
    double ms;
    rc = timed_compress(c, sample, n, p, 1, out, ms);
    if (rc) return fail(rc);
    rc = timed_decompress(c, out, sample, n, 1, back, ms);
    if (rc) return fail(rc);
    out.clear();
  }
  // compressor: CTAs per SM in the persistent form; one chunk per launch in
  // the plain form
  for (int f = 0; f < 2; f++) {
    const int lo = forms[f] == CUCM_FORM_PERSISTENT ? 1 : 0, hi = forms[f] == CUCM_FORM_PERSISTENT ? 2 : 0;
    for (int k = lo; k <= hi; k++) {
      cucm_tune_result r = candidate(forms[f]);
      r.tuning.cmp_ctas = k;
      cucm_ctx_set_tuning(c, &r.tuning);
      rc = timed_compress(c, sample, n, p, reps, ref.empty() ? ref : out, r.compress_ms);
      if (rc) return fail(rc);
      if (!out.empty() && out != ref) return fail(CUCM_EMISMATCH);
      cands.push_back(r);
    }
  }
  {
    // the generic kernel (8 warps per chunk), persistent form
    cucm_tune_result r = candidate(CUCM_FORM_PERSISTENT);
    r.tuning.kernel = 1;
    cucm_ctx_set_tuning(c, &r.tuning);
    rc = timed_compress(c, sample, n, p, reps, out, r.compress_ms);
    if (rc) return fail(rc);
    if (out != ref) return fail(CUCM_EMISMATCH);
    cands.push_back(r);
  }
  // decoder: chunks per CTA and table placement in the persistent form
  for (int f = 0; f < 2; f++) {
    const int max_pairs = forms[f] == CUCM_FORM_PERSISTENT ? 5 : 0;
    for (int dp = 0; dp <= max_pairs; dp++) {
      for (int dt = 0; dt < 2; dt++) {
        cucm_tune_result r = candidate(forms[f]);
        r.tuning.dec_pairs = dp;
        r.tuning.dec_tables = dt;
        cucm_ctx_set_tuning(c, &r.tuning);
        rc = timed_decompress(c, ref, sample, n, reps, back, r.decompress_ms);
        if (rc) return fail(rc);
        cands.push_back(r);
      }
    }
  }
  {
    cucm_tune_result r = candidate(CUCM_FORM_PERSISTENT);
    r.tuning.kernel = 1;
    cucm_ctx_set_tuning(c, &r.tuning);
    rc = timed_decompress(c, ref, sample, n, reps, back, r.decompress_ms);
    if (rc) return fail(rc);
    cands.push_back(r);
  }

  // per form and kernel, the fastest compressor and the fastest decoder
  // choice; the pair with the least sum wins
  double best_total = -1.0;
  for (int f = 0; f < 2; f++) {
    for (int kern = 0; kern < 2; kern++) {
      const cucm_tune_result *bc = nullptr, *bd = nullptr;
      for (const cucm_tune_result &r : cands) {
        if (r.tuning.form != forms[f] || r.tuning.kernel != kern) continue;
        if (r.compress_ms >= 0.0 && (!bc || r.compress_ms < bc->compress_ms)) bc = &r;
        if (r.decompress_ms >= 0.0 && (!bd || r.decompress_ms < bd->decompress_ms)) bd = &r;
      }
      if (!bc || !bd) continue;
      const double total = bc->compress_ms + bd->decompress_ms;
      if (best_total < 0.0 || total < best_total) {
        best_total = total;
        *best = bd->tuning;
        best->cmp_ctas = bc->tuning.cmp_ctas;
      }
    }
  }
  cucm_ctx_set_tuning(c, best);
  for (size_t i = 0; i < cands.size() && i < cap; i++) results[i] = cands[i];
  if (count) *count = (uint32_t)cands.size();
  return CUCM_OK;
}
