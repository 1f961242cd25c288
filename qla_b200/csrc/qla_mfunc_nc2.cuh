// qla_mfunc_nc2.cuh -- the code templates' two-colour closed forms of the
// colour-matrix functions, as engine OPs: compiled into QLA_F2_/QLA_D2_ and
// taken by QLA_FN_/QLA_DN_ at nc = 2, as the templates' `if(NC==2)` branches
// are in both of the reference's builds.
//
//   exp        M_eq_exp_M.c:257-291     (s = tr/2, t = csqrt(-det of a - s),
//                                        c0 = e^s cosh t, c1 = e^s sinh(t)/t)
//   sqrt       M_eq_sqrt_M.c:87-134     (eigenvalues l0, l1; c1 = 1/(sl0+sl1))
//   invsqrt    M_eq_invsqrt_M.c:88-133
//   log        M_eq_log_M.c:103-152
//   expA       M_eq_expA_M.c:312-350    (anti-Hermitian + i*trace)
//   expTA      M_eq_expTA_M.c:301-329   (traceless anti-Hermitian)
//   sqrtPH     M_eq_sqrtPH_M.c:224-262  (positive Hermitian)
//   invsqrtPH  M_eq_invsqrtPH_M.c:228-251
//   det, inverse        C_eq_det_M.c:63-69, M_eq_inverse_M.c:64-78
//   a^-1 b              V_eq_M_inverse_V.c:65-83, M_eq_M_inverse_M.c:65-91
//   eigenvalues         V_eq_eigenvals_M.c:291-296 / V_eq_eigenvalsH_M.c:180-185
//                       (the files' own QLA_eigenvals_2x2)
//
// Every multiply, add and divide is rounded explicitly in the site precision
// R in the order of the complex macros the templates call
// (include/qla_complex.h): QLA_c_eq_r_div_c divides in R, QLA_c_eq_c_div_c
// forms 1.0/|b|^2 in double and rounds it; literals 0.5 are double products
// rounded once.  The complex library functions follow lib/cmath (csqrt,
// cexp, cexpi, clog, csinhcosh).  Results are bit-identical to the reference
// wherever no transcendental function enters (sqrt, invsqrt, sqrtPH,
// invsqrtPH, inverse, det, a^-1 b, eigenvalues); exp, log, expA and expTA
// call CUDA's sinh / exp / sincos / log / atan2 where the reference calls the
// host libm's.  Each OP is a few hundred FP operations on four complex
// numbers: HBM-bound (32 or 64 bytes in, the same out, per site).
#pragma once
#include "qla_mfunc_generic_ext.cuh"

namespace qlab {
namespace nc2 {

using gen::cdiv_q;
using gen::rsqrt_c;
using gen::to_r;

template <typename R>
__device__ __forceinline__ R fabs_r(R x) {
  if constexpr (sizeof(R) == 4) return fabsf(x); else return fabs(x);
}
template <typename R>
__device__ __forceinline__ R copysign_r(R x, R y) {
  if constexpr (sizeof(R) == 4) return copysignf(x, y); else return copysign(x, y);
}
template <typename R>
__device__ __forceinline__ void sincos_q(R x, R* s, R* c) {
  if constexpr (sizeof(R) == 4) sincosf(x, s, c); else sincos(x, s, c);
}

// QLA csqrt (lib/cmath/QLA_csqrt.c): the halvings are double products
template <typename R>
__device__ __forceinline__ Cx<R> csqrt_q(Cx<R> z) {
  const R nrm = rsqrt_c<R>(cnorm2(z));
  const R sr = rsqrt_c<R>(fabs_r(to_r<R>(__dmul_rn(0.5, (double)radd(nrm, z.re)))));
  const R si = copysign_r(rsqrt_c<R>(fabs_r(to_r<R>(__dmul_rn(0.5, (double)rsub(nrm, z.re))))), z.im);
  return Cx<R>{sr, si};
}
// QLA cexp (lib/cmath/QLA_cexp.c): e^re (cos im, sin im)
template <typename R>
__device__ __forceinline__ Cx<R> cexp_q(Cx<R> a) {
  R mag;
  if constexpr (sizeof(R) == 4) mag = expf(a.re); else mag = exp(a.re);
  R s, c;
  sincos_q(a.im, &s, &c);
  return Cx<R>{rmul(mag, c), rmul(mag, s)};
}
// QLA cexpi (lib/cmath/QLA_cexpi.c)
template <typename R>
__device__ __forceinline__ Cx<R> cexpi_q(R t) {
  R s, c;
  sincos_q(t, &s, &c);
  return Cx<R>{c, s};
}
// QLA clog (lib/cmath/QLA_clog.c): 0.5 log|a|^2 in double, atan2 in R
template <typename R>
__device__ __forceinline__ Cx<R> clog_q(Cx<R> a) {
  R arg;
  if constexpr (sizeof(R) == 4) arg = atan2f(a.im, a.re); else arg = atan2(a.im, a.re);
  return Cx<R>{to_r<R>(__dmul_rn(0.5, log((double)cnorm2(a)))), arg};
}
// QLA csinhcosh (lib/cmath/QLA_csinhcosh.c): cosh x = sqrt(1 + sinh^2 x)
template <typename R>
__device__ __forceinline__ void csinhcosh_q(Cx<R> a, Cx<R>& sh, Cx<R>& ch) {
  R sx;
  if constexpr (sizeof(R) == 4) sx = sinhf(a.re); else sx = sinh(a.re);
  const R cx = rsqrt_c<R>(radd(R(1), rmul(sx, sx)));
  R sy, cy;
  sincos_q(a.im, &sy, &cy);
  sh = Cx<R>{rmul(cy, sx), rmul(sy, cx)};
  ch = Cx<R>{rmul(cy, cx), rmul(sy, sx)};
}
// QLA_c_eq_r_div_c with an integer numerator: t = num / |b|^2 in R
template <typename R>
__device__ __forceinline__ Cx<R> rdivc(R num, Cx<R> b) {
  const R t = rdiv(num, cnorm2(b));
  return Cx<R>{rmul(t, b.re), -rmul(t, b.im)};
}
// QLA_c_eq_c_times_c_plus_c: a x + b, left to right
template <typename R>
__device__ __forceinline__ Cx<R> ctcpc(Cx<R> a, Cx<R> x, Cx<R> b) {
  return Cx<R>{radd(rsub(rmul(a.re, x.re), rmul(a.im, x.im)), b.re),
               radd(radd(rmul(a.re, x.im), rmul(a.im, x.re)), b.im)};
}
// QLA_c_eqm_c_times_c: -(a b) as -a.re b.re + a.im b.im, -a.re b.im - a.im b.re
template <typename R>
__device__ __forceinline__ Cx<R> ceqm(Cx<R> a, Cx<R> b) {
  return Cx<R>{radd(-rmul(a.re, b.re), rmul(a.im, b.im)), rsub(-rmul(a.re, b.im), rmul(a.im, b.re))};
}
template <typename R>
__device__ __forceinline__ Cx<R> cadd(Cx<R> a, Cx<R> b) { return Cx<R>{radd(a.re, b.re), radd(a.im, b.im)}; }
template <typename R>
__device__ __forceinline__ Cx<R> csub(Cx<R> a, Cx<R> b) { return Cx<R>{rsub(a.re, b.re), rsub(a.im, b.im)}; }
template <typename R>
__device__ __forceinline__ Cx<R> chalf(Cx<R> a) {  // QLA_c_eq_r_times_c(s, 0.5, a)
  return Cx<R>{to_r<R>(__dmul_rn(0.5, (double)a.re)), to_r<R>(__dmul_rn(0.5, (double)a.im))};
}

// r = c0 + c1 a, complex coefficients
template <typename R>
__device__ __forceinline__ void out_c(Cx<R> (&r)[4], Cx<R> c0, Cx<R> c1, Cx<R> a00, Cx<R> a01, Cx<R> a10, Cx<R> a11) {
  r[0] = ctcpc(c1, a00, c0);
  r[1] = cmul(c1, a01);
  r[2] = cmul(c1, a10);
  r[3] = ctcpc(c1, a11, c0);
}
// r = c0 + c1 a, real coefficients (QLA_c_eq_c_times_r_plus_r, QLA_c_eq_c_times_r)
template <typename R>
__device__ __forceinline__ void out_r(Cx<R> (&r)[4], R c0, R c1, Cx<R> a00, Cx<R> a01, Cx<R> a10, Cx<R> a11) {
  r[0] = Cx<R>{radd(rmul(a00.re, c1), c0), rmul(a00.im, c1)};
  r[1] = Cx<R>{rmul(c1, a01.re), rmul(c1, a01.im)};
  r[2] = Cx<R>{rmul(c1, a10.re), rmul(c1, a10.im)};
  r[3] = Cx<R>{radd(rmul(a11.re, c1), c0), rmul(a11.im, c1)};
}
// Re(a b) - Re(c d): QLA_r_eq_Re_c_times_c then QLA_r_meq_Re_c_times_c
template <typename R>
__device__ __forceinline__ R re_det(Cx<R> a, Cx<R> b, Cx<R> c, Cx<R> d) {
  const R x = rsub(rmul(a.re, b.re), rmul(a.im, b.im));
  return rsub(x, rsub(rmul(c.re, d.re), rmul(c.im, d.im)));
}
template <typename R>
__device__ __forceinline__ Cx<R> det2(const Cx<R> (&a)[4]) {
  Cx<R> det = cmul(a[0], a[3]);
  cmms(det, a[1], a[2]);
  return det;
}

template <typename R>
__device__ void mexp(Cx<R> (&r)[4], const Cx<R> (&a)[4]) {
  const Cx<R> tr = cadd(a[0], a[3]);
  const Cx<R> s = chalf(tr);
  const Cx<R> a00 = csub(a[0], s), a11 = csub(a[3], s);
  Cx<R> mdet = cmul(a[1], a[2]);
  cmms(mdet, a00, a11);
  const Cx<R> t = csqrt_q(mdet);
  Cx<R> st, ch;
  if (t.re == R(0) && t.im == R(0)) {
    st = Cx<R>{R(1), R(0)};
    ch = Cx<R>{R(1), R(0)};
  } else {
    Cx<R> sh;
    csinhcosh_q(t, sh, ch);
    st = cdiv_q(sh, t);
  }
  const Cx<R> es = cexp_q(s);
  out_c(r, cmul(es, ch), cmul(es, st), a00, a[1], a[2], a11);
}

// sqrt (INV false) and invsqrt (INV true) from the eigenvalues l0, l1
template <typename R, bool INV>
__device__ void sqrt2(Cx<R> (&r)[4], const Cx<R> (&a)[4]) {
  Cx<R> l0, l1;
  gen::eig2_g(l0, l1, a[0], a[1], a[2], a[3]);
  const Cx<R> sl0 = csqrt_q(l0), sl1 = csqrt_q(l1);
  const Cx<R> ss = cadd(sl0, sl1);
  Cx<R> ps = cmul(sl0, sl1), c0, c1;
  if constexpr (!INV) {
    if (ss.re == R(0) && ss.im == R(0)) {
      c0 = sl0;
      c1 = Cx<R>{R(0), R(0)};
    } else {
      c1 = rdivc(R(1), ss);
      c0 = cmul(ps, c1);
    }
  } else {
    // the template divides by zero for a singular input
    c1 = rdivc(R(-1), cmul(ps, ss));
    ps = cadd(ps, cadd(a[0], a[3]));
    c0 = ceqm(ps, c1);
  }
  out_c(r, c0, c1, a[0], a[1], a[2], a[3]);
}

template <typename R>
__device__ void mlog(Cx<R> (&r)[4], const Cx<R> (&a)[4]) {
  const Cx<R> s = chalf(cadd(a[0], a[3]));
  const Cx<R> det = det2(a);
  const Cx<R> d = csub(cmul(s, s), det);
  Cx<R> c0, c1;
  if (d.re == R(0) && d.im == R(0)) {
    c0 = Cx<R>{R(0), R(0)};
    c1 = cdiv_q(clog_q(s), s);
  } else {
    const Cx<R> sd = csqrt_q(d);
    const R ts = radd(rmul(s.re, sd.re), rmul(s.im, sd.im));
    Cx<R> e1, de;
    if (ts >= R(0)) {
      e1 = cadd(s, sd);
      de = Cx<R>{rmul(R(2), sd.re), rmul(R(2), sd.im)};
    } else {
      e1 = csub(s, sd);
      de = Cx<R>{rmul(R(-2), sd.re), rmul(R(-2), sd.im)};
    }
    const Cx<R> e0 = cdiv_q(det, e1);
    const Cx<R> le0 = clog_q(e0), le1 = clog_q(e1);
    const Cx<R> dei = rdivc(R(1), de);
    const Cx<R> dl = csub(le1, le0);
    Cx<R> dl0 = cmul(e1, le0);
    cmms(dl0, e0, le1);
    c1 = cmul(dl, dei);
    c0 = cmul(dl0, dei);
  }
  out_c(r, c0, c1, a[0], a[1], a[2], a[3]);
}

// expA (TRACE true: the imaginary part of the trace is kept as a phase) and
// expTA (TRACE false)
template <typename R, bool TRACE>
__device__ void expah2(Cx<R> (&r)[4], const Cx<R> (&a)[4]) {
  if constexpr (TRACE) {
    const Cx<R> s = chalf(cadd(a[0], a[3]));
    const Cx<R> a00 = csub(a[0], s), a11 = csub(a[3], s);
    const R t = rsqrt_c<R>(fabs_r(re_det(a00, a11, a[1], a[2])));
    R st, cs;
    if (t == R(0)) {
      st = R(1);
      cs = R(1);
    } else {
      const Cx<R> sc = cexpi_q(t);
      st = rdiv(sc.im, t);
      cs = sc.re;
    }
    const Cx<R> es = cexpi_q(s.im);
    out_c(r, Cx<R>{rmul(cs, es.re), rmul(cs, es.im)}, Cx<R>{rmul(st, es.re), rmul(st, es.im)}, a00, a[1], a[2], a11);
  } else {
    const R t = rsqrt_c<R>(fabs_r(re_det(a[0], a[3], a[1], a[2])));
    R c0, c1;
    if (t == R(0)) {
      c0 = R(1);
      c1 = R(1);
    } else {
      const Cx<R> sc = cexpi_q(t);
      c0 = sc.re;
      c1 = rdiv(sc.im, t);
    }
    out_r(r, c0, c1, a[0], a[1], a[2], a[3]);
  }
}

// sqrtPH (INV false) and invsqrtPH (INV true)
template <typename R, bool INV>
__device__ void sqrtph2(Cx<R> (&r)[4], const Cx<R> (&a)[4]) {
  const R det = re_det(a[0], a[3], a[1], a[2]);
  const R tr = radd(a[0].re, a[3].re);
  if constexpr (INV) {
    const R sdet = rsqrt_c<R>(fabs_r(det));
    R c1 = rdiv(R(1), rmul(sdet, rsqrt_c<R>(fabs_r(radd(tr, rmul(R(2), sdet))))));
    const R c0 = rmul(radd(tr, sdet), c1);
    c1 = -c1;
    out_r(r, c0, c1, a[0], a[1], a[2], a[3]);
  } else {
    if (det == R(0)) {
      if (tr == R(0)) {
#pragma unroll
        for (int k = 0; k < 4; k++) r[k] = Cx<R>{R(0), R(0)};
      } else {
        const R c1 = rdiv(R(1), rsqrt_c<R>(fabs_r(tr)));
#pragma unroll
        for (int k = 0; k < 4; k++) r[k] = Cx<R>{rmul(c1, a[k].re), rmul(c1, a[k].im)};
      }
    } else {
      const R sdet = rsqrt_c<R>(fabs_r(det));
      const R c1 = rdiv(R(1), rsqrt_c<R>(fabs_r(radd(tr, rmul(R(2), sdet)))));
      out_r(r, rmul(sdet, c1), c1, a[0], a[1], a[2], a[3]);
    }
  }
}

template <typename R>
__device__ __forceinline__ void inverse2(Cx<R> (&x)[4], const Cx<R> (&a)[4]) {
  const Cx<R> idet = rdivc(R(1), det2(a));
  x[0] = cmul(a[3], idet);
  x[1] = ceqm(a[1], idet);
  x[2] = ceqm(a[2], idet);
  x[3] = cmul(a[0], idet);
}

// x = a^-1 b for NB columns of b (NB = 1: ColorVector, 2: ColorMatrix)
template <typename R, int NB>
__device__ __forceinline__ void minv2(Cx<R> (&x)[2 * NB], const Cx<R> (&a)[4], const Cx<R> (&b)[2 * NB]) {
  const Cx<R> idet = rdivc(R(1), det2(a));
#pragma unroll
  for (int j = 0; j < NB; j++) {
    Cx<R> r0 = cmul(a[3], b[j]);
    cmms(r0, a[1], b[NB + j]);
    Cx<R> r1 = cmul(a[0], b[NB + j]);
    cmms(r1, a[2], b[j]);
    x[j] = cmul(r0, idet);
    x[NB + j] = cmul(r1, idet);
  }
}

}  // namespace nc2

enum Nc2Fn { N2_EXP, N2_SQRT, N2_INVSQRT, N2_LOG, N2_EXPA, N2_EXPTA, N2_SQRTPH, N2_INVSQRTPH, N2_INVERSE, N2_DET,
             N2_EIG, N2_EIGH };

// --------------------------------------------------------------- engine OPs
template <typename R_, int FN>
struct Nc2MfuncOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = 4, N1 = 0, N2 = 0,
                       NOUT = FN == N2_DET ? 1 : (FN == N2_EIG || FN == N2_EIGH) ? 2 : 4, NACC = 0;
  __device__ static void apply(const SiteParams&, const Cx<R> (&a)[N0], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               Cx<R> (&r)[NOUT]) {
    if constexpr (FN == N2_EXP) nc2::mexp(r, a);
    else if constexpr (FN == N2_SQRT) nc2::sqrt2<R, false>(r, a);
    else if constexpr (FN == N2_INVSQRT) nc2::sqrt2<R, true>(r, a);
    else if constexpr (FN == N2_LOG) nc2::mlog(r, a);
    else if constexpr (FN == N2_EXPA) nc2::expah2<R, true>(r, a);
    else if constexpr (FN == N2_EXPTA) nc2::expah2<R, false>(r, a);
    else if constexpr (FN == N2_SQRTPH) nc2::sqrtph2<R, false>(r, a);
    else if constexpr (FN == N2_INVSQRTPH) nc2::sqrtph2<R, true>(r, a);
    else if constexpr (FN == N2_INVERSE) nc2::inverse2(r, a);
    else if constexpr (FN == N2_DET) r[0] = nc2::det2(a);
    else if constexpr (FN == N2_EIG) gen::eig2_g(r[0], r[1], a[0], a[1], a[2], a[3]);
    else gen::eig2_h(r[0], r[1], a[0], a[1], a[2], a[3]);
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[N0], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

template <typename R_, int NB>
struct Nc2MInverseOp {
  using R = R_;
  static constexpr int NIN = 2, N0 = 4, N1 = 2 * NB, N2 = 0, NOUT = 2 * NB, NACC = 0;
  __device__ static void apply(const SiteParams&, const Cx<R> (&a)[N0], const Cx<R> (&b)[N1], const Cx<R> (&)[1],
                               Cx<R> (&x)[NOUT]) {
    nc2::minv2<R, NB>(x, a, b);
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[N0], const Cx<R> (&)[N1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

}  // namespace qlab
