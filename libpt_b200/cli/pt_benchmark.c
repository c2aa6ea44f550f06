/*
 * pt_benchmark: the command line of the reference's benchmark program
 * (benchmark.c:348-392), run against this library's pt.h entry points.
 *
 *     pt_benchmark rpt|upt|rft|uft|rptmp|uptmp|rftmp|uftmp o v [ob vb]
 *
 * Fills the host arrays of one solve with uniform random values in
 * [0, 1e-4) (the reference's benchmark.c:40-56 distribution, from its own
 * generator here), calls the entry point once, and prints the energy and
 * the wall time.  Sizes as in the reference: oa = ob = o, va = vb = v,
 * unless ob and vb are given.  Besides the reference's six types it has
 * rftmp and uftmp.  The precision of the FP64 entry points follows
 * LIBPT_FP64_PRECISION, that of the _mp ones LIBPT_MP_PRECISION.
 */
#define _POSIX_C_SOURCE 199309L
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "pt.h"

enum { OV, OOVV, OOVO, OVVV };

/* Elements of one pt.h argument class (src/pt.h:54-178 layouts). */
static size_t class_size(int cls, int unr, size_t oa, size_t va, size_t ob,
                         size_t vb) {
  switch (cls) {
  case OV:
    return oa * va + (unr ? ob * vb : 0);
  case OOVV:
    return oa * oa * va * va + oa * ob * va * vb +
           (unr ? ob * ob * vb * vb + ob * oa * vb * va : 0);
  case OOVO:
    return oa * oa * va * oa + oa * ob * va * ob +
           (unr ? ob * ob * vb * ob + ob * oa * vb * oa : 0);
  default: /* OVVV: packed same-spin blocks */
    return oa * va * (va * (va - 1) / 2) + oa * vb * va * vb +
           (unr ? ob * vb * (vb * (vb - 1) / 2) + ob * va * vb * va : 0);
  }
}

static const int PT_CLASSES[7] = {OV, OV, OV, OOVV, OOVO, OOVV, OVVV};
static const int FT_CLASSES[10] = {OV,   OV,   OV,   OOVV, OOVV,
                                   OOVV, OOVO, OVVV, OOVO, OVVV};

static uint64_t rng_state = 0x243f6a8885a308d3ull;

/* splitmix64: uniform double in [0, 1) */
static double uniform(void) {
  uint64_t z = (rng_state += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  z ^= z >> 31;
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

static void *filled(size_t n, int fp32) {
  void *p = malloc((n ? n : 1) * (fp32 ? sizeof(float) : sizeof(double)));
  if (!p) {
    fprintf(stderr, "pt_benchmark: out of host memory (%zu elements)\n", n);
    exit(1);
  }
  for (size_t i = 0; i < n; ++i) {
    const double x = uniform() / 10000.0;
    if (fp32)
      ((float *)p)[i] = (float)x;
    else
      ((double *)p)[i] = x;
  }
  return p;
}

int main(int argc, char **argv) {
  static const char *types[8] = {"rpt",   "upt",   "rft",   "uft",
                                 "rptmp", "uptmp", "rftmp", "uftmp"};
  if (argc != 4 && argc != 6) {
    fprintf(stderr, "usage: pt_benchmark rpt|upt|rft|uft|rptmp|uptmp|rftmp|"
                    "uftmp o v [ob vb]\n");
    return 1;
  }
  int t = -1;
  for (int i = 0; i < 8; ++i)
    if (strcmp(argv[1], types[i]) == 0) t = i;
  if (t < 0) {
    fprintf(stderr, "pt_benchmark: bad benchmark type '%s'\n", argv[1]);
    return 1;
  }
  const int ft = (t & 3) >= 2, unr = t & 1, mp = t >= 4;
  const size_t oa = strtoull(argv[2], NULL, 10), va = strtoull(argv[3], NULL, 10);
  const size_t ob = argc == 6 ? strtoull(argv[4], NULL, 10) : oa;
  const size_t vb = argc == 6 ? strtoull(argv[5], NULL, 10) : va;
  printf("%s, oa = %zu, va = %zu, ob = %zu, vb = %zu\n", argv[1], oa, va, ob,
         vb);

  const int nargs = ft ? 10 : 7;
  const int *cls = ft ? FT_CLASSES : PT_CLASSES;
  void *a[10];
  double gb = 0.0;
  for (int i = 0; i < nargs; ++i) {
    const size_t n = class_size(cls[i], unr, oa, va, ob, vb);
    gb += (double)n * (mp ? 4 : 8) / 1e9;
    a[i] = filled(n, mp);
  }
  printf("inputs: %.3f GB (host)\n", gb);

  struct timespec t0, t1;
  clock_gettime(CLOCK_MONOTONIC, &t0);
  double e = 0.0;
#define D(i) ((const double *)a[i])
#define F(i) ((const float *)a[i])
  switch (t) {
  case 0: e = libpt_rpt(oa, va, D(0), D(1), D(2), D(3), D(4), D(5), D(6)); break;
  case 1:
    e = libpt_upt(oa, va, ob, vb, D(0), D(1), D(2), D(3), D(4), D(5), D(6));
    break;
  case 2:
    e = libpt_rft(oa, va, D(0), D(1), D(2), D(3), D(4), D(5), D(6), D(7), D(8),
                  D(9));
    break;
  case 3:
    e = libpt_uft(oa, va, ob, vb, D(0), D(1), D(2), D(3), D(4), D(5), D(6),
                  D(7), D(8), D(9));
    break;
  case 4:
    e = libpt_rpt_mp(oa, va, F(0), F(1), F(2), F(3), F(4), F(5), F(6));
    break;
  case 5:
    e = libpt_upt_mp(oa, va, ob, vb, F(0), F(1), F(2), F(3), F(4), F(5), F(6));
    break;
  case 6:
    e = libpt_rft_mp(oa, va, F(0), F(1), F(2), F(3), F(4), F(5), F(6), F(7),
                     F(8), F(9));
    break;
  default:
    e = libpt_uft_mp(oa, va, ob, vb, F(0), F(1), F(2), F(3), F(4), F(5), F(6),
                     F(7), F(8), F(9));
    break;
  }
#undef D
#undef F
  clock_gettime(CLOCK_MONOTONIC, &t1);
  const double sec = (double)(t1.tv_sec - t0.tv_sec) +
                     1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
  printf("energy = %.17g\n", e);
  printf("done in %.3f sec\n", sec);
  for (int i = 0; i < nargs; ++i) free(a[i]);
  return 0;
}
