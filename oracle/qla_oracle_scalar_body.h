/*
 * Test infrastructure (the oracle) -- NOT product code.
 * The real / complex / integer field libraries QLA_F_ / QLA_D_ restated from
 * the loops the reference generator emits (lib/perl/build_qla.pl:186-355,
 * 1936-2082, 2089-2555; include/qla_complex.h:110-140, 417-428 for norm, arg
 * and division; lib/cmath/QLA_cexp.c, QLA_cexpi.c, QLA_clog.c, QLA_csqrt.c
 * for the complex functions), with the host libm as the reference uses it.
 * Op codes follow the product's ScalarOp enumeration.  Included twice by
 * qla_oracle_scalar.c (R = float with the float libm names for QLA_F_, R =
 * double for QLA_D_).
 */
#define CAT2_(a, b) a##_##b
#define CAT2(a, b) CAT2_(a, b)
#define FN(name) CAT2(name, SFX)

typedef struct { R re, im; } FN(zc);

static R FN(ldr)(const void *p, const int *ix, long k) { return ((const R *)p)[ix ? ix[k] : k]; }
static int FN(ldi)(const void *p, const int *ix, long k) { return ((const int *)p)[ix ? ix[k] : k]; }
static FN(zc) FN(ldc)(const void *p, const int *ix, long k) { return ((const FN(zc) *)p)[ix ? ix[k] : k]; }

static R FN(math1)(int op, R x)
{
  switch (op) {
  case 18: return MSIN(x);
  case 19: return MCOS(x);
  case 20: return MTAN(x);
  case 21: return MASIN(x);
  case 22: return MACOS(x);
  case 23: return MATAN(x);
  case 24: return MSQRT(x);
  case 25: return MFABS(x);
  case 26: return MEXP(x);
  case 27: return MLOG(x);
  case 28: return MLOG10(x);
  case 29: return MSINH(x);
  case 30: return MCOSH(x);
  case 31: return MTANH(x);
  case 32: return MCEIL(x);
  default: return MFLOOR(x);
  }
}

/* r[k] (eqop)= op(a, b, c, s) over the sites k = gang[i] (or i); pointer forms
 * gather through idx_*; s is the real constant of the r_times / fill forms */
void FN(ora_scalar)(int op, int eqop, void *r, const void *a, const void *b, const void *c, R s, long n,
                    const int *ia, const int *ib, const int *ic, const int *gang)
{
  for (long i = 0; i < n; i++) {
    const long k = gang ? gang[i] : i;
    if (op <= 38) {
      R *o = (R *)r + k, t = 0;
      switch (op) {
      case 0: t = FN(ldr)(a, ia, k); break;
      case 1: t = FN(ldr)(a, ia, k) * FN(ldr)(b, ib, k); break;
      case 2: t = s * FN(ldr)(b, ib, k); break;
      case 3: t = s; break;
      case 4: *o = 0.; continue;
      case 5: if (FN(ldi)(b, ib, k)) *o = FN(ldr)(a, ia, k); continue;
      case 6: *o = FN(ldi)(a, ia, k); continue;
      case 7: *o = FN(ldr)(a, ia, k) + FN(ldr)(b, ib, k); continue;
      case 8: *o = FN(ldr)(a, ia, k) - FN(ldr)(b, ib, k); continue;
      case 9: *o = FN(ldr)(a, ia, k) / FN(ldr)(b, ib, k); continue;
      case 10: { R x = FN(ldr)(a, ia, k), y = FN(ldr)(b, ib, k); *o = (x > y ? x : y); continue; }
      case 11: { R x = FN(ldr)(a, ia, k), y = FN(ldr)(b, ib, k); *o = (x > y ? y : x); continue; }
      case 12: *o = fmod(FN(ldr)(a, ia, k), FN(ldr)(b, ib, k)); continue;
      case 13: *o = pow(FN(ldr)(a, ia, k), FN(ldr)(b, ib, k)); continue;
      case 14: *o = atan2(FN(ldr)(a, ia, k), FN(ldr)(b, ib, k)); continue;
      case 15: *o = ldexp(FN(ldr)(a, ia, k), FN(ldi)(b, ib, k)); continue;
      case 16: *o = s * FN(ldr)(b, ib, k) + FN(ldr)(c, ic, k); continue;
      case 17: *o = s * FN(ldr)(b, ib, k) - FN(ldr)(c, ic, k); continue;
      case 34: *o = FN(ldr)(a, ia, k) >= 0 ? 1. : -1.; continue;
      case 35: *o = FN(ldc)(a, ia, k).re; continue;
      case 36: *o = FN(ldc)(a, ia, k).im; continue;
      case 37: { FN(zc) z = FN(ldc)(a, ia, k); *o = MSQRT(z.re * z.re + z.im * z.im); continue; }
      case 38: { FN(zc) z = FN(ldc)(a, ia, k); *o = MATAN2(z.im, z.re); continue; }
      default: *o = FN(math1)(op, FN(ldr)(a, ia, k)); continue;
      }
      if (eqop == 0) *o = t;
      else if (eqop == 1) *o += t;
      else if (eqop == 2) *o -= t;
      else *o = -t;
    } else if (op <= 46) {
      int *o = (int *)r + k;
      R x = FN(ldr)(a, ia, k);
      switch (op) {
      case 39: *o = (x == FN(ldr)(b, ib, k)); break;
      case 40: *o = (x >= FN(ldr)(b, ib, k)); break;
      case 41: *o = (x > FN(ldr)(b, ib, k)); break;
      case 42: *o = (x <= FN(ldr)(b, ib, k)); break;
      case 43: *o = (x < FN(ldr)(b, ib, k)); break;
      case 44: *o = (x != FN(ldr)(b, ib, k)); break;
      case 45: *o = MROUND(x); break;
      default: *o = x; break;
      }
    } else {
      FN(zc) *o = (FN(zc) *)r + k;
      switch (op) {
      case 47: o->re = FN(ldr)(a, ia, k); o->im = 0; break;
      case 48: o->re = FN(ldr)(a, ia, k); o->im = FN(ldr)(b, ib, k); break;
      case 49: {
        FN(zc) x = FN(ldc)(a, ia, k), y = FN(ldc)(b, ib, k);
        R t = 1.0 / (y.re * y.re + y.im * y.im);
        o->re = (x.re * y.re + x.im * y.im) * t;
        o->im = (x.im * y.re - x.re * y.im) * t;
        break;
      }
      case 50: {
        FN(zc) x = FN(ldc)(a, ia, k);
        R mag = MEXP(x.re), sn, cs;
        MSINCOS(x.im, &sn, &cs);
        o->re = mag * cs; o->im = mag * sn;
        break;
      }
      case 51: { R sn, cs; MSINCOS(FN(ldr)(a, ia, k), &sn, &cs); o->re = cs; o->im = sn; break; }
      case 52: {
        FN(zc) x = FN(ldc)(a, ia, k);
        o->re = 0.5 * log(x.re * x.re + x.im * x.im);
        o->im = MATAN2(x.im, x.re);
        break;
      }
      default: {
        FN(zc) x = FN(ldc)(a, ia, k);
        R nn = MSQRT(x.re * x.re + x.im * x.im), rr = x.re, ii = x.im;
        R sr = MSQRT(MFABS(0.5 * (nn + rr)));
        R si = MCOPYSIGN(MSQRT(MFABS(0.5 * (nn - rr))), ii);
        o->re = sr; o->im = si;
        break;
      }
      }
    }
  }
}

/* global reductions of real / integer fields in the reference's order, one
 * double sum: kind 0 a.b, 1 |a|^2, 2 sum a; isint: the fields are QLA_Int */
double FN(ora_sred)(int kind, int isint, const void *a, const void *b, long n, const int *ia, const int *ib,
                    const int *gang)
{
  double sum = 0.;
  for (long i = 0; i < n; i++) {
    const long k = gang ? gang[i] : i;
    if (isint) {
      const int x = FN(ldi)(a, ia, k);
      if (kind == 0) sum += (int)((unsigned)x * (unsigned)FN(ldi)(b, ib, k));
      else if (kind == 1) { R at = x; sum += (at) * (at); }
      else sum += x;
    } else {
      const R x = FN(ldr)(a, ia, k);
      if (kind == 0) sum += x * FN(ldr)(b, ib, k);
      else if (kind == 1) { R at = x; sum += (at) * (at); }
      else sum += x;
    }
  }
  return sum;
}

#undef FN
#undef CAT2
#undef CAT2_
