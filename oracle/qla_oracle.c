/*
 * Test infrastructure (the oracle) -- NOT product code.
 *
 * A CPU restatement of the QLA 1.9.0 level-1 operators on the B200 hot path,
 * used only by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg
 * as the checker.  The product library (qla_b200/) never links or calls it.
 *
 * Pinning: tests/test_oracle_pin.py checks this restatement against golden
 * vectors produced by the reference library itself (tests/golden/, written by
 * tests/golden/make_golden.py from oracle/_ref/libqla_ref.so, which
 * oracle/build_ref.sh builds from the reference's own generator output), and,
 * when oracle/_ref is present, against that library directly on larger
 * seeded inputs.  Linear ops are expected bit-identical; reductions agree to
 * the reference's own rounding.
 *
 * Build: oracle/Makefile  ->  oracle/liboracle.so  (gcc -O2 -ffp-contract=off).
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>
#include "qla_oracle.h"

#define R float
#define SFX f
#include "qla_oracle_body.h"
#undef R
#undef SFX

#define R double
#define SFX d
#include "qla_oracle_body.h"
#undef R
#undef SFX

/* ------------------------------------------------------------------------ */
/* Extended-precision reductions (the "FP64 in question" oracle).  QLA itself
 * has no extended reduction (QLA_QD3 sums in double, datatypes.pl:357-358), so
 * this restates the check of test/src/protocol_tensor_sng.m4:1209-1222
 * (chkNorm2, accumulating in QLA_Q_Real) with double-double arithmetic:
 * TwoProduct via fma and Knuth's TwoSum, which keeps ~106 bits. */
typedef struct { double hi, lo; } dd_t;

static inline void dd_add(dd_t *s, double x)
{
  double t = s->hi + x;
  double bp = t - s->hi;
  double err = (s->hi - (t - bp)) + (x - bp);
  s->hi = t;
  s->lo += err;
}

static inline void dd_add_prod(dd_t *s, double a, double b)
{
  double p = a * b;
  double e = fma(a, b, -p);
  dd_add(s, p);
  dd_add(s, e);
}

static inline long site_(const int *gang, long i) { return gang ? gang[i] : i; }
static inline long rec_(const int *idx, long k) { return idx ? idx[k] : k; }

#define DEF_EXACT(SFXN, RT)                                                        \
double ora_norm2_exact_##SFXN(const RT *a, long n, int ncplx,                      \
                              const int *idx_a, const int *gang)                   \
{                                                                                  \
  dd_t s = {0., 0.};                                                               \
  for (long i = 0; i < n; i++) {                                                   \
    long k = site_(gang, i);                                                       \
    const RT *A = a + 2 * rec_(idx_a, k) * ncplx;                                  \
    for (int e = 0; e < 2 * ncplx; e++) dd_add_prod(&s, A[e], A[e]);               \
  }                                                                                \
  return s.hi + s.lo;                                                              \
}                                                                                  \
void ora_dot_exact_##SFXN(double *out2, const RT *a, const RT *b, long n,          \
                          int ncplx, const int *idx_a, const int *idx_b,           \
                          const int *gang)                                         \
{                                                                                  \
  dd_t sr = {0., 0.}, si = {0., 0.};                                               \
  for (long i = 0; i < n; i++) {                                                   \
    long k = site_(gang, i);                                                       \
    const RT *A = a + 2 * rec_(idx_a, k) * ncplx;                                  \
    const RT *B = b + 2 * rec_(idx_b, k) * ncplx;                                  \
    for (int e = 0; e < ncplx; e++) {                                              \
      double ar = A[2*e], ai = A[2*e+1], br = B[2*e], bi = B[2*e+1];               \
      dd_add_prod(&sr, ar, br); dd_add_prod(&sr, ai, bi);                          \
      dd_add_prod(&si, ar, bi); dd_add_prod(&si, -ai, br);                         \
    }                                                                              \
  }                                                                                \
  out2[0] = sr.hi + sr.lo; out2[1] = si.hi + si.lo;                                \
}

DEF_EXACT(f, float)
DEF_EXACT(d, double)

int ora_version(void) { return 1; }
