/*
 * Test infrastructure (the oracle) -- NOT product code.
 * QLA's per-site random-number generator restated from lib/random:
 * QLA_random.c:18-36 (shift register xor congruential generator),
 * QLA_gaussian.c:19-55 (Box-Muller; MILC's polar method when the milc flag
 * is set, the spare deviate kept in the addend / scale words),
 * QLA_seed_random.c:13-36; and the vectorised fills, seeding and state copies
 * the generator emits from them (lib/perl/build_qla.pl:2620-2690,
 * 2058-2084, 370-400), in the reference's site and element order.
 */
#include <math.h>

#include "qla_oracle.h"

typedef struct {
  unsigned int r0, r1, r2, r3, r4, r5, r6;
  unsigned int multiplier, addend, ic_state;
  float scale;
} ora_rs;

float ora_rng_uniform(void *pv)
{
  ora_rs *p = (ora_rs *)pv;
  int t = (((p->r5 >> 7) | (p->r6 << 17)) ^ ((p->r4 >> 1) | (p->r5 << 23))) & 0xffffff;
  p->r6 = p->r5;
  p->r5 = p->r4;
  p->r4 = p->r3;
  p->r3 = p->r2;
  p->r2 = p->r1;
  p->r1 = p->r0;
  p->r0 = t;
  unsigned int s = p->ic_state * p->multiplier + 12345u;
  p->ic_state = s;
  return (1.0f / ((float)0x1000000)) * (float)(t ^ (int)((s >> 8) & 0xffffffu));
}

float ora_rng_gaussian(void *rsv, int milc)
{
  ora_rs *rs = (ora_rs *)rsv;
  if (milc) {
    if (rs->addend != 0) {
      rs->addend = 0;
      double v1, v2, rsq;
      do {
        v1 = (double)ora_rng_uniform(rs);
        v2 = (double)ora_rng_uniform(rs);
        v1 = 2.0 * v1 - 1.0;
        v2 = 2.0 * v2 - 1.0;
        rsq = v1 * v1 + v2 * v2;
      } while ((rsq >= 1.0) || (rsq == 0.0));
      double fac = sqrt(-2.0 * log(rsq) / rsq);
      rs->scale = (float)(v1 * fac);
      return (float)(v2 * fac);
    }
    rs->addend = 1;
    return rs->scale;
  }
  double v, p, r;
  v = ora_rng_uniform(rs);
  p = ora_rng_uniform(rs) * 2. * 3.14159265358979323846;
  r = sqrt(2. * (-log(v + 1e-307)));
  return (float)(r * cos(p));
}

void ora_rng_seed(void *pv, int seed, int index)
{
  ora_rs *p = (ora_rs *)pv;
  unsigned int m = 69607u + 8u * (unsigned int)index, x = (unsigned int)seed;
  unsigned int *w[7] = {&p->r0, &p->r1, &p->r2, &p->r3, &p->r4, &p->r5, &p->r6};
  for (int j = 0; j < 7; j++) {
    x = m * x + 12345u;
    *w[j] = (x >> 8) & 0xffffff;
  }
  x = m * x + 12345u;
  p->ic_state = x;
  p->multiplier = 100005u + 8u * (unsigned int)index;
  p->addend = 12345;
  p->scale = 1.0 / ((float)0x1000000);
}

/* r[k] (nreal reals) = uniform (gauss 0) or gaussian deviates from state
 * s[ks]; states gathered through idx_s (pointer forms) */
#define ORA_RNG_FILL(R, SFX)                                                                     \
void ora_rng_fill_##SFX(int nreal, int gauss, int milc, R *r, void *s, long n, const int *idx_s, \
                        const int *gang)                                                         \
{                                                                                                \
  ora_rs *S = (ora_rs *)s;                                                                       \
  for (long i = 0; i < n; i++) {                                                                 \
    const long k = gang ? gang[i] : i;                                                           \
    ora_rs *st = &S[idx_s ? idx_s[k] : k];                                                       \
    for (int c = 0; c < nreal; c++)                                                              \
      r[k * nreal + c] = gauss ? ora_rng_gaussian(st, milc) : ora_rng_uniform(st);               \
  }                                                                                              \
}
ORA_RNG_FILL(float, f)
ORA_RNG_FILL(double, d)

void ora_rng_seedfield(void *r, int seed, const int *a, long n, const int *idx_a, const int *gang)
{
  ora_rs *S = (ora_rs *)r;
  for (long i = 0; i < n; i++) {
    const long k = gang ? gang[i] : i;
    ora_rng_seed(&S[k], seed, a[idx_a ? idx_a[k] : k]);
  }
}

void ora_rng_copy(void *r, const void *a, const int *mask, long n, const int *idx_a, const int *idx_m,
                  const int *gang)
{
  ora_rs *R = (ora_rs *)r;
  const ora_rs *A = (const ora_rs *)a;
  for (long i = 0; i < n; i++) {
    const long k = gang ? gang[i] : i;
    if (mask && !mask[idx_m ? idx_m[k] : k]) continue;
    R[k] = A[idx_a ? idx_a[k] : k];
  }
}
