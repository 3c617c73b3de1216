/*
 * workload_gen.c -- seeded synthetic inputs for benchmarks and tests.
 *
 * The byte-serial parts of the generators (the order-2 Markov text chain
 * with forced word breaks) are too slow in Python, so they live here; the
 * transition tables themselves are drawn in numpy (cucm_b200/workloads.py).
 * Random numbers: splitmix64.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>

static inline uint64_t sm64(uint64_t *s) {
  uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static inline double unit_open(uint64_t *s) { /* (0, 1) */
  return ((double)(sm64(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

/* Geometric on {1, 2, ...} with success probability p. */
static inline uint64_t geometric(uint64_t *s, double p) {
  double u = unit_open(s);
  return (uint64_t)floor(log(u) / log1p(-p)) + 1;
}

/*
 * Order-2 Markov text over `nsym` symbols.  cdf[(a * nsym + b) * nsym + c]
 * is the cumulative probability (scaled to 2^32) of next symbol c after
 * symbols (a, b); sym[] maps symbol index to byte.  A space (symbol
 * `space_idx`) is forced whenever the current word length, drawn from
 * geometric(p_word), runs out.
 */
void wl_markov_text(const uint32_t *cdf, const uint8_t *sym, int nsym, int space_idx, double p_word,
                    uint64_t seed, uint8_t *out, uint64_t n) {
  uint64_t s = seed;
  int a = space_idx, b = space_idx;
  uint64_t word = geometric(&s, p_word);
  for (uint64_t i = 0; i < n; i++) {
    int c;
    if (word == 0) {
      c = space_idx;
      word = geometric(&s, p_word);
    } else {
      const uint32_t *row = cdf + ((size_t)a * nsym + b) * nsym;
      uint32_t u = (uint32_t)(sm64(&s) >> 32);
      int lo = 0, hi = nsym - 1;
      while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (u < row[mid]) hi = mid; else lo = mid + 1;
      }
      c = lo;
      word--;
    }
    out[i] = sym[c];
    a = b;
    b = c;
  }
}
