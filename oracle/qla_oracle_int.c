/*
 * Test infrastructure (the oracle) -- NOT product code.
 * QLA_I_ integer site operations restated from the reference's integer
 * library (lib/perl/build_qla.pl:1932-2082): r[k] (eqop) f(a, b, c, *s) with
 * C's int semantics (the generated code is plain C on int).
 * code: see ora_int_value; eqop 0 eq, 1 peq, 2 meq, 3 eqm; mask keeps r.
 * Index arrays model `pI` pointer operands (a[k] = *pa[k] = src[idx[k]]) and
 * the gang index of the `x` variants.
 */
#include <stddef.h>
#include "qla_oracle.h"

static int ora_int_value(int code, int a, int b, int c, int s)
{
  (void)c;
  switch (code) {
  case 0: return a;                                  /* copy */
  case 1: return (int)((unsigned)a * (unsigned)b);   /* times (wraps as on x86) */
  case 2: return (int)((unsigned)a + (unsigned)b);   /* plus */
  case 3: return (int)((unsigned)a - (unsigned)b);   /* minus */
  case 4: return a / b;                              /* divide */
  case 5: return a % b;                              /* mod */
  case 6: return a & b;
  case 7: return a | b;
  case 8: return a ^ b;
  case 9: return (int)((unsigned)a << b);            /* lshift */
  case 10: return a >> b;                            /* rshift (arithmetic) */
  case 11: return a == b;
  case 12: return a != b;
  case 13: return a < b;
  case 14: return a <= b;
  case 15: return a > b;
  case 16: return a >= b;
  case 17: return a > b ? a : b;                     /* max */
  case 18: return a < b ? a : b;                     /* min */
  case 20: return !a;                                /* not */
  case 21: return 0;                                 /* zero */
  case 22: return s;                                 /* r = *s */
  case 23: return (int)((unsigned)s * (unsigned)a);  /* *s * a */
  case 24: return (int)((unsigned)s * (unsigned)a + (unsigned)b);
  default: return (int)((unsigned)s * (unsigned)a - (unsigned)b);
  }
}

void ora_int(int code, int eqop, int *r, const int *a, const int *b, const int *c, int s, long n,
             const int *ia, const int *ib, const int *ic, const int *gang)
{
  for (long i = 0; i < n; i++) {
    long k = gang ? gang[i] : i;
    int av = a ? a[ia ? ia[k] : k] : 0;
    int bv = b ? b[ib ? ib[k] : k] : 0;
    int cv = c ? c[ic ? ic[k] : k] : 0;
    if (code == 19) {                                /* mask: if (b) r = a */
      if (bv) r[k] = av;
      continue;
    }
    int v = ora_int_value(code, av, bv, cv, s);
    switch (eqop) {
    case 0: r[k] = v; break;
    case 1: r[k] = (int)((unsigned)r[k] + (unsigned)v); break;
    case 2: r[k] = (int)((unsigned)r[k] - (unsigned)v); break;
    default: r[k] = (int)(0u - (unsigned)v); break;
    }
  }
}
