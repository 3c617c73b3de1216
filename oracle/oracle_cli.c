/*
 * oracle_cli.c -- command-line driver for the CPU restatement (test
 * infrastructure only).
 *   oracle_cli c IN OUT CHUNKSIZE UNIT PRELEARN BATCH [THREADS]
 *   oracle_cli d IN OUT [THREADS]
 */
#include <stdio.h>
#include <stdlib.h>

#include "cucm_oracle.h"

static unsigned char *slurp(const char *path, size_t *n) {
  FILE *f = fopen(path, "rb");
  if (!f) return NULL;
  fseek(f, 0, SEEK_END);
  long sz = ftell(f);
  fseek(f, 0, SEEK_SET);
  unsigned char *b = (unsigned char *)malloc(sz ? (size_t)sz : 1);
  if (b && fread(b, 1, (size_t)sz, f) != (size_t)sz) {
    free(b);
    b = NULL;
  }
  fclose(f);
  *n = (size_t)sz;
  return b;
}

int main(int argc, char **argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: %s c IN OUT CS UNIT PRELEARN BATCH [THREADS] | d IN OUT [THREADS]\n", argv[0]);
    return 2;
  }
  size_t n;
  unsigned char *in = slurp(argv[2], &n);
  if (!in) {
    fprintf(stderr, "cannot read %s\n", argv[2]);
    return 1;
  }
  unsigned char *out = NULL;
  size_t out_n = 0;
  int rc;
  if (argv[1][0] == 'c') {
    if (argc < 8) return 2;
    int threads = argc > 8 ? atoi(argv[8]) : 0;
    rc = co_compress(in, n, strtoull(argv[4], 0, 10), atoi(argv[5]), strtoull(argv[6], 0, 10),
                     atoi(argv[7]), threads, &out, &out_n);
  } else {
    int threads = argc > 4 ? atoi(argv[4]) : 0;
    rc = co_decompress(in, n, threads, &out, &out_n);
  }
  if (rc != 0) {
    fprintf(stderr, "error %d\n", rc);
    return 1;
  }
  FILE *f = fopen(argv[3], "wb");
  if (!f || fwrite(out, 1, out_n, f) != out_n) return 1;
  fclose(f);
  printf("%zu -> %zu\n", n, out_n);
  return 0;
}
