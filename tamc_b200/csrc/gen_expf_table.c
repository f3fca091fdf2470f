// gen_expf_table.c -- build step: writes the exception table that makes
// tamc_expf_exact() return glibc's expf bits for every float argument.
//
// It compares tamc_expf_core(x) with the host libm expf(x) for every float x in
// [0, 89] and [-110, -0] (about 2.2e9 arguments, a few seconds on 8 cores) and
// writes, little-endian:
//   u32 magic 'EXPT', u32 nbuckets, u32 nentries,
//   u32 off[nbuckets + 1], u32 keys[nentries], u32 vals[nentries]
// It also checks that outside that range both functions agree on a sample.
// Usage: gen_expf_table <out.bin>
#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "expf_exact.h"

typedef struct { uint32_t k, v; } ent_t;

static int cmp_ent(const void* a, const void* b) {
  uint32_t x = ((const ent_t*)a)->k, y = ((const ent_t*)b)->k;
  return x < y ? -1 : x > y;
}

static void scan(uint32_t lo, uint32_t hi, ent_t** out, size_t* n, size_t* cap) {
  const int nt = omp_get_max_threads();
  ent_t** loc = calloc((size_t)nt, sizeof(ent_t*));
  size_t* ln = calloc((size_t)nt, sizeof(size_t));
  size_t* lc = calloc((size_t)nt, sizeof(size_t));
#pragma omp parallel
  {
    const int t = omp_get_thread_num();
#pragma omp for schedule(static, 1 << 20)
    for (long long b = lo; b <= (long long)hi; ++b) {
      const float x = tamc_u2f((uint32_t)b);
      const float g = expf(x);
      const float c = tamc_expf_core(x);
      if (tamc_f2u(g) != tamc_f2u(c)) {
        if (ln[t] == lc[t]) {
          lc[t] = lc[t] ? 2 * lc[t] : 4096;
          loc[t] = realloc(loc[t], lc[t] * sizeof(ent_t));
        }
        loc[t][ln[t]].k = (uint32_t)b;
        loc[t][ln[t]].v = tamc_f2u(g);
        ln[t]++;
      }
    }
  }
  for (int t = 0; t < nt; ++t) {
    if (*n + ln[t] > *cap) {
      *cap = (*n + ln[t]) * 2;
      *out = realloc(*out, *cap * sizeof(ent_t));
    }
    if (ln[t]) memcpy(*out + *n, loc[t], ln[t] * sizeof(ent_t));
    *n += ln[t];
    free(loc[t]);
  }
  free(loc); free(ln); free(lc);
}

int main(int argc, char** argv) {
  if (argc != 2) { fprintf(stderr, "usage: %s out.bin\n", argv[0]); return 2; }
  ent_t* e = NULL;
  size_t n = 0, cap = 0;
  scan(0u, TAMC_EXPF_POS_MAX_BITS, &e, &n, &cap);
  scan(0x80000000u, TAMC_EXPF_NEG_MAX_BITS, &e, &n, &cap);
  qsort(e, n, sizeof(ent_t), cmp_ent);
  // outside the scanned range both must give inf / 0 / NaN consistently
  for (uint32_t b = TAMC_EXPF_POS_MAX_BITS + 1; b < 0x7f800000u; b += 977) {
    float x = tamc_u2f(b);
    if (tamc_f2u(expf(x)) != tamc_f2u(tamc_expf_core(x))) { fprintf(stderr, "range check failed (+)\n"); return 1; }
  }
  for (uint32_t b = TAMC_EXPF_NEG_MAX_BITS + 1; b < 0xff800000u; b += 977) {
    float x = tamc_u2f(b);
    if (tamc_f2u(expf(x)) != tamc_f2u(tamc_expf_core(x))) { fprintf(stderr, "range check failed (-)\n"); return 1; }
  }
  const uint32_t nb = TAMC_EXPF_NUM_BUCKETS;
  uint32_t* off = calloc((size_t)nb + 1, 4);
  size_t i = 0;
  for (uint32_t bk = 0; bk < nb; ++bk) {
    off[bk] = (uint32_t)i;
    while (i < n) {
      uint32_t b;
      tamc_expf_bucket(e[i].k, &b);
      if (b != bk) break;
      ++i;
    }
  }
  off[nb] = (uint32_t)i;
  if (i != n) { fprintf(stderr, "bucket walk mismatch\n"); return 1; }
  FILE* f = fopen(argv[1], "wb");
  if (!f) { perror("open"); return 1; }
  const uint32_t hdr[3] = {0x54505845u, nb, (uint32_t)n};
  fwrite(hdr, 4, 3, f);
  fwrite(off, 4, (size_t)nb + 1, f);
  for (size_t k = 0; k < n; ++k) fwrite(&e[k].k, 4, 1, f);
  for (size_t k = 0; k < n; ++k) fwrite(&e[k].v, 4, 1, f);
  fclose(f);
  printf("expf exception table: %zu entries, %u buckets\n", n, nb);
  free(off); free(e);
  return 0;
}
