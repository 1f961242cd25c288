// qla_mfunc_ext.cuh -- the remaining Nc = 3 colour-matrix functions of the
// reference's code templates, as engine OPs:
//
//   M = a^-1 b, V = a^-1 b    M_eq_M_inverse_M.c:85-135 (Gauss-Jordan, every
//                             nc > 2), V_eq_M_inverse_V.c:84-126 (Cramer)
//   invsqrt                   M_eq_invsqrt_M.c:88-127 (Newton)
//   log                       M_eq_log_M.c:127-199 (4 square roots + rational)
//   expTA, expA               M_eq_expTA_M.c:96-274, M_eq_expA_M.c:100-298
//                             (Cayley-Hamilton closed form)
//   sqrtPH, invsqrtPH         M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201
//   eigenvalsH, eigenvals     V_eq_eigenvalsH_M.c:106-166,
//                             V_eq_eigenvals_M.c:127-186 (cubic roots)
//   reunit (no counterpart)   u (u^+ u)^(-1/2) from the pieces above
//
// Precision.  a^-1 b uses only +, -, *, / and is evaluated in the site
// precision with explicitly rounded operations: bit-identical to QLA_F3 and
// QLA_D3.  invsqrt and log run the templates' Newton iteration and rational
// approximation in the site precision too (the templates' own arithmetic:
// float matrices with double norms for F3), so they equal QLA_F3's and
// QLA_D3's results except where CUDA's log of |a|_F and the host libm's
// differ in the last place.  The closed forms are evaluated in FP64 for both
// F3 and D3 -- the coefficients of the cubic and the closed-form
// coefficients near degenerate eigenvalues are where FP32 loses digits --
// in the templates' operation order with explicitly rounded FP64 arithmetic,
// and the F3 result is rounded once to float; the closed forms
// call acos, sincos, cbrt, pow and atan2, whose CUDA and host-libm results
// may differ by an ulp, so D3 agrees with QLA_D3 to a few ulps away from
// the templates' branch points.
#pragma once
#include "qla_mfunc.cuh"
#include "qla_ops.cuh"

namespace qlab {

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// QLA_D_cexpi (lib/cmath/QLA_cexpi.c:22-30)
__device__ __forceinline__ Cx<double> cexpi(double t) {
  double s, c;
  sincos(t, &s, &c);
  return Cx<double>{c, s};
}

template <typename R>
__device__ __forceinline__ void promote9(Cx<double> (&d)[9], const Cx<R> (&a)[9]) {
#pragma unroll
  for (int k = 0; k < 9; k++) d[k] = cd(a[k]);
}
template <typename R, int N>
__device__ __forceinline__ void round_out(Cx<R> (&r)[N], const Cx<double> (&d)[N]) {
#pragma unroll
  for (int k = 0; k < N; k++) r[k] = cround<R>(d[k]);
}

// r = a * b, each element as the templates' local `mul` macro writes it:
// x = a_i0 b_0j, then x += a_i1 b_1j, x += a_i2 b_2j
__device__ __forceinline__ void mat3_mul_first(Cx<double> (&r)[9], const Cx<double> (&a)[9],
                                               const Cx<double> (&b)[9]) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      Cx<double> x = cmul(a[i * 3], b[j]);
      cpms(x, a[i * 3 + 1], b[3 + j]);
      cpms(x, a[i * 3 + 2], b[6 + j]);
      r[i * 3 + j] = x;
    }
}

// m += s * a (QLA_D3_M_peq_r_times_M)
__device__ __forceinline__ void m_peq_r_m(Cx<double> (&m)[9], double s, const Cx<double> (&a)[9]) {
#pragma unroll
  for (int k = 0; k < 9; k++) m[k] = Cx<double>{dadd(m[k].re, dmul(s, a[k].re)), dadd(m[k].im, dmul(s, a[k].im))};
}
// m = d 1 (QLA_D3_M_eq_c with a real constant)
__device__ __forceinline__ void m_eq_d(Cx<double> (&m)[9], double d) {
#pragma unroll
  for (int k = 0; k < 9; k++) m[k] = Cx<double>{(k % 4 == 0) ? d : 0.0, 0.0};
}
// the three 2x2 cofactors used by every 3x3 closed form
template <typename R>
__device__ __forceinline__ void cofactors3(Cx<R>& det0, Cx<R>& det1, Cx<R>& det2, const Cx<R> (&a)[9]) {
  det2 = cmul(a[0], a[4]);
  cmms(det2, a[1], a[3]);
  det1 = cmul(a[2], a[3]);
  cmms(det1, a[0], a[5]);
  det0 = cmul(a[1], a[5]);
  cmms(det0, a[2], a[4]);
}

// ---------------------------------------------------------------------------
// r = a^-1 b, site precision.  NB = 1: ColorVector (Cramer's rule);
// NB = 3: ColorMatrix (Gauss-Jordan).
template <typename R_, int NB>
struct MInverseOp {
  using R = R_;
  static constexpr int NIN = 2, N0 = 9, N1 = 3 * NB, N2 = 0, NOUT = 3 * NB, NACC = 0;
  __device__ __forceinline__ static void apply(const SiteParams&, const Cx<R> (&a)[9], const Cx<R> (&b)[N1],
                                               const Cx<R> (&)[1], Cx<R> (&x)[NOUT]) {
    if constexpr (NB == 1) {
      Cx<R> det0, det1, det2;
      cofactors3(det0, det1, det2, a);
      Cx<R> det = cmul(det2, a[8]);
      cpms(det, det1, a[7]);
      cpms(det, det0, a[6]);
      const R t = rdiv(R(1), cnorm2(det));
      const Cx<R> idet{rmul(t, det.re), rmul(-t, det.im)};
      Cx<R> r[3] = {cmul(det0, b[2]), cmul(det1, b[2]), cmul(det2, b[2])};
#define QLAB_SETV(i0, j0, i1, j1, i2, j2)              \
  {                                                    \
    Cx<R> d_ = cmul(a[i1 * 3 + j1], a[i2 * 3 + j2]);   \
    cmms(d_, a[i1 * 3 + j2], a[i2 * 3 + j1]);          \
    cpms(r[i0], d_, b[j0]);                            \
  }
      QLAB_SETV(0, 0, 1, 1, 2, 2);
      QLAB_SETV(0, 1, 2, 1, 0, 2);
      QLAB_SETV(1, 0, 1, 2, 2, 0);
      QLAB_SETV(1, 1, 2, 2, 0, 0);
      QLAB_SETV(2, 0, 1, 0, 2, 1);
      QLAB_SETV(2, 1, 2, 0, 0, 1);
#undef QLAB_SETV
#pragma unroll
      for (int i = 0; i < 3; i++) x[i] = cmul(r[i], idet);
    } else {
      Cx<R> c[9];
#pragma unroll
      for (int k = 0; k < 9; k++) c[k] = a[k];
#pragma unroll
      for (int k = 0; k < NOUT; k++) x[k] = b[k];
      gj_solve3<R, NB>(c, x);
    }
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[9], const Cx<R> (&)[N1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

// ---------------------------------------------------------------------------
// M_eq_invsqrt_M: x = 1, e = 0.5 |a|_F a^-1 - 0.5, Newton, r = x / sqrt|a|_F,
// in the site precision (double scalars enter as (R)(0.5 ds) and
// (R)(1/sqrt ds), as the template's M_eq_d_times_M does)
template <typename R_>
struct InvsqrtOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = 9, N1 = 0, N2 = 0, NOUT = 9, NACC = 0;
  __device__ static void apply(const SiteParams&, const Cx<R> (&a)[9], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               Cx<R> (&r)[9]) {
    double ds = fnorm2_3(a);
    if (ds == 0.0) {  // M_eq_d(r, 1./0.)
#pragma unroll
      for (int k = 0; k < 9; k++) r[k] = Cx<R>{(k % 4 == 0) ? R(INFINITY) : R(0), R(0)};
      return;
    }
    ds = __dsqrt_rn(ds);
    Cx<R> xi[9], x[9], e[9];
    inv3(xi, a);
    const R hds = (R)dmul(0.5, ds);
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const bool dg = (k % 4 == 0);
      e[k] = Cx<R>{radd(dg ? R(-0.5) : R(0), rmul(hds, xi[k].re)), radd(R(0), rmul(hds, xi[k].im))};
      x[k] = Cx<R>{radd(dg ? R(1) : R(0), e[k].re), radd(R(0), e[k].im)};
    }
    newton_sqrt3(x, e);
    const R rr = (R)ddiv(1.0, __dsqrt_rn(ds));
#pragma unroll
    for (int k = 0; k < 9; k++) r[k] = Cx<R>{rmul(rr, x[k].re), rmul(rr, x[k].im)};
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[9], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

// m += s * a (QLA_<P>3_M_peq_r_times_M) and m = d 1 (QLA_<P>3_M_eq_c with a
// real constant) in the site precision
template <typename R>
__device__ __forceinline__ void m_peq_r_m_site(Cx<R> (&m)[9], R s, const Cx<R> (&a)[9]) {
#pragma unroll
  for (int k = 0; k < 9; k++) m[k] = Cx<R>{radd(m[k].re, rmul(s, a[k].re)), radd(m[k].im, rmul(s, a[k].im))};
}
template <typename R>
__device__ __forceinline__ void m_eq_d_site(Cx<R> (&m)[9], R d) {
#pragma unroll
  for (int k = 0; k < 9; k++) m[k] = Cx<R>{(k % 4 == 0) ? d : R(0), R(0)};
}

// ---------------------------------------------------------------------------
// M_eq_log_M: as = a/|a|_F, four square roots, log(1+x) with the template's
// rational coefficients, times 16, plus log|a|_F on the diagonal -- in the
// site precision (the coefficients enter as (R)P, (R)Q; log|a|_F is added in
// double and rounded, as `r += ds` does with a double ds)
template <typename R_>
struct LogOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = 9, N1 = 0, N2 = 0, NOUT = 9, NACC = 0;
  __device__ static void apply(const SiteParams&, const Cx<R> (&a)[9], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               Cx<R> (&r)[9]) {
    constexpr double P0 = 7.70838733755885391666E0, P1 = 1.79368678507819816313E1,
                     P2 = 1.44989225341610930846E1, P3 = 4.70579119878881725854E0,
                     P4 = 4.97494994976747001425E-1, P5 = 1.01875663804580931796E-4;
    constexpr double Q0 = 2.31251620126765340583E1, Q1 = 7.11544750618563894466E1,
                     Q2 = 8.29875266912776603211E1, Q3 = 4.52279145837532221105E1,
                     Q4 = 1.12873587189167450590E1;
    Cx<R> as[9], t[9];
    double ds = __dsqrt_rn(fnorm2_3(a));
    if (ds == 0.0) {  // M_eq_d(r, log(0))
#pragma unroll
      for (int k = 0; k < 9; k++) r[k] = Cx<R>{(k % 4 == 0) ? R(-INFINITY) : R(0), R(0)};
      return;
    }
    const R rr = (R)ddiv(1.0, ds);
#pragma unroll
    for (int k = 0; k < 9; k++) as[k] = Cx<R>{rmul(rr, a[k].re), rmul(rr, a[k].im)};
#pragma unroll 1
    for (int i = 0; i < 4; i++) {
#pragma unroll
      for (int k = 0; k < 9; k++) t[k] = as[k];
      sqrt3(as, t);
    }
#pragma unroll
    for (int i = 0; i < 3; i++) as[i * 4].re = rsub(as[i * 4].re, R(1));
    Cx<R> pa[9], qa[9], as2[9], as3[9];
    m_eq_d_site(pa, (R)P0);
    m_eq_d_site(qa, (R)Q0);
    m_peq_r_m_site(pa, (R)P1, as);
    m_peq_r_m_site(qa, (R)Q1, as);
    mat3_mul(as2, as, as);
    m_peq_r_m_site(pa, (R)P2, as2);
    m_peq_r_m_site(qa, (R)Q2, as2);
    mat3_mul(as3, as, as2);
    m_peq_r_m_site(pa, (R)P3, as3);
    m_peq_r_m_site(qa, (R)Q3, as3);
    mat3_mul(t, as2, as2);  // as4
    m_peq_r_m_site(pa, (R)P4, t);
    m_peq_r_m_site(qa, (R)Q4, t);
    {
      Cx<R> as5[9];
      mat3_mul(as5, as, t);
      m_peq_r_m_site(pa, (R)P5, as5);
#pragma unroll
      for (int k = 0; k < 9; k++) qa[k] = Cx<R>{radd(qa[k].re, as5[k].re), radd(qa[k].im, as5[k].im)};
    }
    inv3(t, qa);        // as5 = qa^-1
    mat3_mul(qa, pa, t);
    mat3_mul(pa, as3, qa);
    m_peq_r_m_site(pa, R(-0.5), as2);
#pragma unroll
    for (int k = 0; k < 9; k++) pa[k] = Cx<R>{radd(pa[k].re, as[k].re), radd(pa[k].im, as[k].im)};
    ds = log(ds);
#pragma unroll
    for (int k = 0; k < 9; k++) {
      Cx<R> v{rmul(R(16), pa[k].re), rmul(R(16), pa[k].im)};
      if (k % 4 == 0) v.re = (R)dadd((double)v.re, ds);
      r[k] = v;
    }
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[9], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

// ---------------------------------------------------------------------------
// exp of a traceless anti-Hermitian i Q: eigenvalues of Q from
// x^3 - p2/2 x - det = 0, exp(iQ) = f0 + f1 (iQ) + f2 (iQ)^2
// (getfs of M_eq_expTA_M.c:139-216; the same function in M_eq_expA_M.c)
__device__ __forceinline__ void getfs_exp(Cx<double>& f0, Cx<double>& f1, Cx<double>& f2, double p2, double det) {
  const double q = dmul(1. / 6., p2);
  const double r = dmul(-0.5, det);
  const double sq = __dsqrt_rn(fabs(q));
  const double sq3 = dmul(dmul(sq, sq), sq);
  if (sq3 > fabs(r)) {
    const double t = acos(ddiv(r, sq3));
    const Cx<double> sct = cexpi(dmul(1. / 3., t));
    const double sqc = dmul(sq, sct.re);
    const double sqs = dmul(dmul(1.73205080756887729352, sq), sct.im);
    const double l0 = dmul(-2.0, sqc);
    const double l1 = dadd(sqc, sqs);
    const double l2 = dsub(sqc, sqs);
    const double d10 = dmul(0.5, dsub(l1, l0));
    const double d20 = dmul(0.5, dsub(l2, l0));
    const double d21 = dsub(l2, l1);
    const Cx<double> eis01 = cexpi(dmul(0.5, dadd(l0, l1)));
    Cx<double> eid10, g10, eid20, eis02, g20;
    if (d10 == 0.0) {
      eid10 = Cx<double>{1.0, 0.0};
      g10 = eis01;
    } else {
      eid10 = cexpi(d10);
      const double sc10 = ddiv(eid10.im, d10);
      g10 = Cx<double>{dmul(sc10, eis01.re), dmul(sc10, eis01.im)};
    }
    const Cx<double> ff0{dadd(dmul(eis01.re, eid10.re), dmul(eis01.im, eid10.im)),
                         dsub(dmul(eis01.im, eid10.re), dmul(eis01.re, eid10.im))};
    if (d20 == 0.0) {
      eis02 = ff0;
      g20 = eis02;
    } else {
      eid20 = cexpi(d20);
      eis02 = cmul(ff0, eid20);
      const double sc20 = ddiv(eid20.im, d20);
      g20 = Cx<double>{dmul(sc20, eis02.re), dmul(sc20, eis02.im)};
    }
    const Cx<double> g2010{dsub(g20.re, g10.re), dsub(g20.im, g10.im)};
    Cx<double> b2{0.0, 0.0};
    if (d21 != 0.0) {
      const double d21i = ddiv(1.0, d21);
      b2 = Cx<double>{dmul(d21i, g2010.re), dmul(d21i, g2010.im)};
    }
    f2 = Cx<double>{b2.im, -b2.re};
    const double m01 = -dadd(l0, l1);
    f1 = Cx<double>{dadd(dmul(m01, b2.re), g10.re), dadd(dmul(m01, b2.im), g10.im)};
    const Cx<double> f10{-g10.im, g10.re};
    const Cx<double> z{dadd(dmul(l1, f2.re), f10.re), dadd(dmul(l1, f2.im), f10.im)};
    f0 = Cx<double>{dadd(dmul(-l0, z.re), ff0.re), dadd(dmul(-l0, z.im), ff0.im)};
  } else if (r == 0.0) {  // zero matrix
    f0 = f1 = f2 = Cx<double>{0.0, 0.0};
  } else {
    const double a = -cbrt(r);
    const Cx<double> eia2 = cexpi(dmul(0.5, a));
    const Cx<double> eia = cmul(eia2, eia2);
    const Cx<double> ei3a2 = cmul(eia, eia2);
    const double snc = ddiv(ei3a2.im, dmul(1.5, a));
    const Cx<double> t{dmul(snc, eia2.re), dmul(snc, eia2.im)};
    f1 = Cx<double>{-t.im, t.re};
    f2 = Cx<double>{0.0, 0.0};
    f0 = cmul(eia2, Cx<double>{ei3a2.re, dmul(-1. / 3., ei3a2.im)});
  }
}

// TRACE = false: expTA (M_eq_expTA_M.c:218-274); TRACE = true: expA
// (M_eq_expA_M.c:222-298) removes i Im(tr)/3 from the diagonal first and
// multiplies the coefficients by exp(i Im(tr)/3)
template <typename R_, bool TRACE>
struct ExpAHOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = 9, N1 = 0, N2 = 0, NOUT = 9, NACC = 0;
  __device__ static void apply(const SiteParams&, const Cx<R> (&a)[9], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               Cx<R> (&r)[9]) {
    Cx<double> iq[9], mqq[9];
    promote9(iq, a);
    Cx<double> f{1.0, 0.0};
    if constexpr (TRACE) {
      const double tr = dadd(dadd(iq[0].im, iq[4].im), iq[8].im);
      const double s = dmul(1. / 3., tr);
      iq[0].im = dsub(iq[0].im, s);
      iq[4].im = dsub(iq[4].im, s);
      iq[8].im = dsub(iq[8].im, s);
      f = cexpi(s);
    }
    mat3_mul_first(mqq, iq, iq);
    const double p2 = dsub(dsub(-mqq[0].re, mqq[4].re), mqq[8].re);
    Cx<double> det0, det1, det2;
    cofactors3(det0, det1, det2, iq);
    double det = dsub(dmul(-det2.re, iq[8].im), dmul(det2.im, iq[8].re));
    det = dsub(det, dadd(dmul(det1.re, iq[7].im), dmul(det1.im, iq[7].re)));
    det = dsub(det, dadd(dmul(det0.re, iq[6].im), dmul(det0.im, iq[6].re)));
    Cx<double> a0, a1, a2;
    getfs_exp(a0, a1, a2, p2, det);
    if constexpr (TRACE) {
      a0 = cmul(f, a0);
      a1 = cmul(f, a1);
      a2 = cmul(f, a2);
    }
#pragma unroll
    for (int k = 0; k < 9; k++) {
      Cx<double> e = cmul(a2, mqq[k]);
      cpms(e, a1, iq[k]);
      if (k % 4 == 0) e = Cx<double>{dadd(e.re, a0.re), dadd(e.im, a0.im)};
      r[k] = cround<R>(e);
    }
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[9], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

// ---------------------------------------------------------------------------
// sqrt (INV = false) or inverse sqrt (INV = true) of a positive Hermitian
// matrix as f0 + f1 m + f2 m^2 from the roots of
// x^3 - tr x^2 + (tr^2 - p2)/2 x - det = 0
// (getfs of M_eq_sqrtPH_M.c:84-138, M_eq_invsqrtPH_M.c:84-142)
template <bool INV>
__device__ __forceinline__ void getfs_sqrtph(double& f0, double& f1, double& f2, double tr, double p2,
                                             double det) {
  const double tr3 = dmul(1. / 3., tr);
  const double p23 = dmul(1. / 3., p2);
  const double tr32 = dmul(tr3, tr3);
  const double q = dmul(0.5, dsub(p23, tr32));
  const double r = dsub(dmul(dmul(0.25, tr3), dsub(dmul(5.0, tr32), p2)), dmul(0.5, det));
  const double sq = __dsqrt_rn(fabs(q));
  const double sq3 = dmul(dmul(sq, sq), sq);
  if (sq3 > fabs(r)) {
    const double t = acos(ddiv(r, sq3));
    const Cx<double> sct = cexpi(dmul(1. / 3., t));
    const double sqc = dmul(sq, sct.re);
    const double sqs = dmul(dmul(1.73205080756887729352, sq), sct.im);
    const double l0 = dsub(tr3, dmul(2.0, sqc));
    const double ll = dadd(tr3, sqc);
    const double l1 = dadd(ll, sqs);
    const double l2 = dsub(ll, sqs);
    const double sl0 = __dsqrt_rn(fabs(l0));
    const double sl1 = __dsqrt_rn(fabs(l1));
    const double sl2 = __dsqrt_rn(fabs(l2));
    const double u = dadd(dadd(sl0, sl1), sl2);
    const double w = dmul(dmul(sl0, sl1), sl2);
    if constexpr (!INV) {
      const double v = dadd(dmul(sl0, dadd(sl1, sl2)), dmul(sl1, sl2));
      const double d = dmul(dmul(dadd(sl0, sl1), dadd(sl0, sl2)), dadd(sl1, sl2));
      const double di = ddiv(1.0, d);
      f0 = dmul(dmul(u, w), di);
      f1 = dmul(dadd(tr, v), di);
      f2 = -di;
    } else {
      const double d = dmul(dmul(dmul(w, dadd(sl0, sl1)), dadd(sl0, sl2)), dadd(sl1, sl2));
      const double di = ddiv(1.0, d);
      const double s = dadd(dadd(dadd(dmul(dmul(w, u), u), dmul(dmul(l0, sl0), dadd(l1, l2))),
                                 dmul(dmul(l1, sl1), dadd(l0, l2))),
                            dmul(dmul(l2, sl2), dadd(l0, l1)));
      f0 = dmul(s, di);
      f1 = dmul(-dadd(dmul(tr, u), w), di);
      f2 = dmul(u, di);
    }
  } else if (r == 0.0) {  // all eigenvalues equal to tr/3
    f0 = INV ? ddiv(1.0, __dsqrt_rn(fabs(tr3))) : __dsqrt_rn(fabs(tr3));
    f1 = 0.0;
    f2 = 0.0;
  } else {
    const double a = -cbrt(r);
    const double l0 = dadd(tr3, dmul(2.0, a));
    const double l1 = dsub(tr3, a);
    const double sl0 = __dsqrt_rn(fabs(l0));
    const double sl1 = __dsqrt_rn(fabs(l1));
    const double sl01 = dadd(sl0, sl1);
    f2 = 0.0;
    if constexpr (!INV) {
      f1 = (sl01 == 0.0) ? 0.0 : ddiv(1.0, sl01);
      f0 = dmul(dmul(sl0, sl1), f1);
    } else {
      const double p01 = dmul(sl0, sl1);
      const double ti = ddiv(1.0, dmul(p01, sl01));
      f1 = -ti;
      f0 = dmul(dadd(dadd(p01, l0), l1), ti);
    }
  }
}

// f0 + f1 m + f2 m^2 of a positive Hermitian m (M_eq_sqrtPH_M.c:140-197,
// M_eq_invsqrtPH_M.c:144-201)
template <bool INV>
__device__ __forceinline__ void sqrtph3_fp64(Cx<double> (&r)[9], const Cx<double> (&m)[9]) {
  Cx<double> mm[9];
  const double tr = dadd(dadd(m[0].re, m[4].re), m[8].re);
  mat3_mul_first(mm, m, m);
  const double p2 = dadd(dadd(mm[0].re, mm[4].re), mm[8].re);
  Cx<double> det0, det1, det2;
  cofactors3(det0, det1, det2, m);
  double det = dsub(dmul(det2.re, m[8].re), dmul(det2.im, m[8].im));
  det = dadd(det, dsub(dmul(det1.re, m[7].re), dmul(det1.im, m[7].im)));
  det = dadd(det, dsub(dmul(det0.re, m[6].re), dmul(det0.im, m[6].im)));
  double f0, f1, f2;
  getfs_sqrtph<INV>(f0, f1, f2, tr, p2, det);
#pragma unroll
  for (int k = 0; k < 9; k++) {
    Cx<double> e{dmul(f2, mm[k].re), dmul(f2, mm[k].im)};
    e = Cx<double>{dadd(e.re, dmul(f1, m[k].re)), dadd(e.im, dmul(f1, m[k].im))};
    if (k % 4 == 0) e.re = dadd(e.re, f0);
    r[k] = e;
  }
}

template <typename R_, bool INV>
struct SqrtPHOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = 9, N1 = 0, N2 = 0, NOUT = 9, NACC = 0;
  __device__ static void apply(const SiteParams&, const Cx<R> (&a)[9], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               Cx<R> (&r)[9]) {
    Cx<double> m[9], y[9];
    promote9(m, a);
    sqrtph3_fp64<INV>(y, m);
    round_out(r, y);
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[9], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

// Unitarity reprojection r = u (u^+ u)^(-1/2), with no counterpart in the
// reference: the composition QLA_D3_M_eq_Ma_times_M -> M_eq_invsqrtPH_M ->
// M_eq_M_times_M evaluated in FP64 with those functions' operation order,
// fused so that u is read once and r written once.
template <typename R_>
struct ReunitOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = 9, N1 = 0, N2 = 0, NOUT = 9, NACC = 0;
  __device__ static void apply(const SiteParams&, const Cx<R> (&a)[9], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               Cx<R> (&r)[9]) {
    Cx<double> u[9], t[9], s[9];
    promote9(u, a);
    lmult_site<double, 3, 3, true, false>(EQ, false, u, u, t);   // u^+ u
    sqrtph3_fp64<true>(s, t);                                     // (u^+ u)^(-1/2)
    lmult_site<double, 3, 3, false, false>(EQ, false, u, s, t);  // u s
    round_out(r, t);
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[9], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

// ---------------------------------------------------------------------------
// eigenvalues of a Hermitian matrix (V_eq_eigenvalsH_M.c:106-166)
template <typename R_>
struct EigenvalsHOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = 9, N1 = 0, N2 = 0, NOUT = 3, NACC = 0;
  __device__ static void apply(const SiteParams&, const Cx<R> (&ain)[9], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               Cx<R> (&v)[3]) {
    Cx<double> m[9];
    promote9(m, ain);
    Cx<double> a00 = m[0], a11 = m[4], a22 = m[8];
    const double s1 = dmul(1. / 3., dadd(dadd(a00.re, a11.re), a22.re));
    a00.re = dsub(a00.re, s1);
    a11.re = dsub(a11.re, s1);
    a22.re = dsub(a22.re, s1);
    Cx<double> det2 = cmul(a00, a11);
    cmms(det2, m[1], m[3]);
    Cx<double> det1 = cmul(m[2], m[3]);
    cmms(det1, a00, m[5]);
    Cx<double> det0 = cmul(m[1], m[5]);
    cmms(det0, m[2], a11);
    double det = dsub(dmul(det2.re, a22.re), dmul(det2.im, a22.im));
    det = dadd(det, dsub(dmul(det1.re, m[7].re), dmul(det1.im, m[7].im)));
    det = dadd(det, dsub(dmul(det0.re, m[6].re), dmul(det0.im, m[6].im)));
    double s2 = det2.re;
    s2 = dadd(s2, dsub(dmul(a00.re, a22.re), dmul(a00.im, a22.im)));
    s2 = dsub(s2, dsub(dmul(m[2].re, m[6].re), dmul(m[2].im, m[6].im)));
    s2 = dadd(s2, dsub(dmul(a11.re, a22.re), dmul(a11.im, a22.im)));
    s2 = dsub(s2, dsub(dmul(m[5].re, m[7].re), dmul(m[5].im, m[7].im)));
    const double q = dmul(-1. / 3., s2);
    const double r = dmul(-0.5, det);
    const double sq = __dsqrt_rn(fabs(q));
    const double sq3 = dmul(dmul(sq, sq), sq);
    double e0, e1, e2;
    if (sq3 > fabs(r)) {
      const double t = acos(ddiv(r, sq3));
      const Cx<double> sct = cexpi(dmul(1. / 3., t));
      const double sqc = dmul(sq, sct.re);
      const double sqs = dmul(dmul(1.73205080756887729352, sq), sct.im);
      e0 = dsub(s1, dmul(2.0, sqc));
      const double ee = dadd(s1, sqc);
      e1 = dadd(ee, sqs);
      e2 = dsub(ee, sqs);
    } else {
      const double a = -cbrt(r);
      e0 = dadd(s1, dmul(2.0, a));
      e1 = dsub(s1, a);
      e2 = e1;
    }
    v[0] = Cx<R>{(R)e0, R(0)};
    v[1] = Cx<R>{(R)e1, R(0)};
    v[2] = Cx<R>{(R)e2, R(0)};
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[9], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

// QLA_D_csqrt, QLA_D_cpow (lib/cmath/QLA_csqrt.c:50-62, QLA_cpow.c:49-58)
__device__ __forceinline__ Cx<double> csqrt_d(Cx<double> z) {
  const double n = __dsqrt_rn(cnorm2(z));
  const double sr = __dsqrt_rn(fabs(dmul(0.5, dadd(n, z.re))));
  const double si = copysign(__dsqrt_rn(fabs(dmul(0.5, dsub(n, z.re)))), z.im);
  return Cx<double>{sr, si};
}
__device__ __forceinline__ Cx<double> cpow_d(Cx<double> a, double b) {
  const double r = pow(cnorm2(a), dmul(0.5, b));
  const Cx<double> c = cexpi(dmul(b, atan2(a.im, a.re)));
  return Cx<double>{dmul(r, c.re), dmul(r, c.im)};
}

// eigenvalues of a general complex matrix (V_eq_eigenvals_M.c:127-186)
template <typename R_>
struct EigenvalsOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = 9, N1 = 0, N2 = 0, NOUT = 3, NACC = 0;
  __device__ static void apply(const SiteParams&, const Cx<R> (&ain)[9], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               Cx<R> (&v)[3]) {
    Cx<double> m[9];
    promote9(m, ain);
    Cx<double> a00 = m[0], a11 = m[4], a22 = m[8];
    Cx<double> s1{dadd(a00.re, a11.re), dadd(a00.im, a11.im)};
    s1 = Cx<double>{dadd(s1.re, a22.re), dadd(s1.im, a22.im)};
    s1 = Cx<double>{dmul(1. / 3., s1.re), dmul(1. / 3., s1.im)};
    a00 = Cx<double>{dsub(a00.re, s1.re), dsub(a00.im, s1.im)};
    a11 = Cx<double>{dsub(a11.re, s1.re), dsub(a11.im, s1.im)};
    a22 = Cx<double>{dsub(a22.re, s1.re), dsub(a22.im, s1.im)};
    Cx<double> det2 = cmul(a00, a11);
    cmms(det2, m[1], m[3]);
    Cx<double> det1 = cmul(m[2], m[3]);
    cmms(det1, a00, m[5]);
    Cx<double> det0 = cmul(m[1], m[5]);
    cmms(det0, m[2], a11);
    Cx<double> det = cmul(det2, a22);
    cpms(det, det1, m[7]);
    cpms(det, det0, m[6]);
    Cx<double> s2 = det2;
    cpms(s2, a00, a22);
    cmms(s2, m[2], m[6]);
    cpms(s2, a11, a22);
    cmms(s2, m[5], m[7]);
    const Cx<double> p{dmul(1. / 3., s2.re), dmul(1. / 3., s2.im)};
    Cx<double> q{dmul(-0.5, det.re), dmul(-0.5, det.im)};
    const Cx<double> p2 = cmul(p, p);
    const Cx<double> q2 = cmul(q, q);
    const Cx<double> d{dadd(dsub(dmul(p.re, p2.re), dmul(p.im, p2.im)), q2.re),
                       dadd(dadd(dmul(p.re, p2.im), dmul(p.im, p2.re)), q2.im)};
    const Cx<double> t = csqrt_d(d);
    const double ts = dadd(dmul(q.re, t.re), dmul(q.im, t.im));
    if (ts >= 0.0)
      q = Cx<double>{dadd(q.re, t.re), dadd(q.im, t.im)};
    else
      q = Cx<double>{dsub(q.re, t.re), dsub(q.im, t.im)};
    const Cx<double> w0 = cpow_d(q, 1. / 3.);
    const Cx<double> w{-0.5, 0.86602540378443864676};
    Cx<double> pw0{0.0, 0.0};
    {  // safedivC(&pw0, &p, &w0, 0)
      const double dd = cnorm2(w0);
      if (dd != 0.0) {
        const double di = ddiv(1.0, dd);
        pw0 = Cx<double>{dadd(dmul(p.re, w0.re), dmul(p.im, w0.im)), dsub(dmul(p.im, w0.re), dmul(p.re, w0.im))};
        pw0 = Cx<double>{dmul(di, pw0.re), dmul(di, pw0.im)};
      }
    }
    const Cx<double> e0{dsub(pw0.re, w0.re), dsub(pw0.im, w0.im)};
    Cx<double> e1{dadd(dmul(w.re, pw0.re), dmul(w.im, pw0.im)), dsub(dmul(w.re, pw0.im), dmul(w.im, pw0.re))};
    cmms(e1, w, w0);
    Cx<double> e2 = cmul(w, pw0);
    e2 = Cx<double>{dsub(e2.re, dadd(dmul(w.re, w0.re), dmul(w.im, w0.im))),
                    dsub(e2.im, dsub(dmul(w.re, w0.im), dmul(w.im, w0.re)))};
    v[0] = cround<R>(Cx<double>{dadd(s1.re, e0.re), dadd(s1.im, e0.im)});
    v[1] = cround<R>(Cx<double>{dadd(s1.re, e1.re), dadd(s1.im, e1.im)});
    v[2] = cround<R>(Cx<double>{dadd(s1.re, e2.re), dadd(s1.im, e2.im)});
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[9], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

}  // namespace qlab
