// qla_mfunc_generic_ext.cuh -- the remaining matrix functions of the code
// templates for a compile-time colour count NC (QLA_FN_ at nc = NC).
//
// Generic paths, restated in the site precision R with explicitly rounded
// operations in the templates' order (bit-identical to the reference's
// N-colour build; log up to the last place of the host libm's log):
//   a^-1 b     V_eq_M_inverse_V.c:128-168, M_eq_M_inverse_M.c:85-135
//              (Gauss-Jordan; NC = 3 with a vector uses Cramer's rule, :84-126)
//   invsqrt    M_eq_invsqrt_M.c:88-127 (Newton from a^-1)
//   log        M_eq_log_M.c:127-199 (four Newton square roots + rational form)
//   eigenvalues V_eq_eigenvalsH_M.c:195-483 = V_eq_eigenvals_M.c:306-594
//              (Hessenberg reduction with pivoting, implicit double-shift QR,
//              2x2 blocks by the template's own 2x2 formula)
// For NC = 3 the templates' closed forms (expA, expTA, sqrtPH, invsqrtPH,
// eigenvalues) are the Nc = 3 OPs of qla_mfunc_ext.cuh; for NC != 3,
// expA / expTA take the exp path and sqrtPH / invsqrtPH the Newton paths,
// as the templates do.
#pragma once
#include "qla_mfunc_ext.cuh"
#include "qla_mfunc_generic.cuh"

namespace qlab {
namespace gen {

// x = a^-1 b for NB right-hand-side columns (Gauss-Jordan with a row
// permutation, the templates' arithmetic)
template <typename R, int NC, int NB>
__device__ void solve_nb(Cx<R> (&x)[NC * NB], const Mat<R, NC>& a, const Cx<R> (&b)[NC * NB]) {
  Mat<R, NC> c = a;
  Cx<R> d[NC * NB];
  for (int k = 0; k < NC * NB; k++) d[k] = b[k];
  int row[NC];
#pragma unroll
  for (int i = 0; i < NC; i++) row[i] = i;
  for (int k = 0; k < NC; k++) {
    R rmax = cnorm2(c(row[k], k));
    int imax = k;
    for (int i = k + 1; i < NC; i++) {
      const R rr = cnorm2(c(row[i], k));
      if (rr > rmax) {
        rmax = rr;
        imax = i;
      }
    }
    {
      const int rk = row[k];
      row[k] = row[imax];
      row[imax] = rk;
    }
    rmax = rdiv(R(1), rmax);
    const int rkk = row[k];
    const Cx<R> s{rmul(rmax, c(rkk, k).re), -rmul(rmax, c(rkk, k).im)};
    c(rkk, k) = s;
    for (int i = 0; i < NC; i++) {
      if (i == k) continue;
      const int ri = row[i];
      const Cx<R> t = cmul(s, c(ri, k));
      for (int j = k + 1; j < NC; j++) cmms(c(ri, j), t, c(rkk, j));
      for (int j = 0; j < NB; j++) cmms(d[ri * NB + j], t, d[rkk * NB + j]);
    }
  }
  for (int i = 0; i < NC; i++)
    for (int j = 0; j < NB; j++) x[i * NB + j] = cmul(c(row[i], i), d[row[i] * NB + j]);
}

// M_eq_inverse_M: NC = 3 cofactors, else Gauss-Jordan against 1
template <typename R, int NC>
__device__ __forceinline__ void inverse_any(Mat<R, NC>& x, const Mat<R, NC>& a) {
  if constexpr (NC == 3) {
    inv3(x.e, a.e);
  } else {
    Mat<R, NC> one;
    m_eq_d(one, R(1));
    m_eq_m_inverse_m(x, a, one);
  }
}

// Newton loop shared by sqrt and invsqrt (FLT/DBL_EPSILON, 20 iterations)
template <typename R, int NC>
__device__ void newton_loop(Mat<R, NC>& x, Mat<R, NC>& e) {
  const double eps = sizeof(R) == 4 ? 1.1920928955078125e-07 : 2.220446049250313080847e-16;
  Mat<R, NC> t1, t2;
  int nit = 0;
  double enorm;
  do {
    nit++;
    m_eq_m_inverse_m(t1, x, e);
    m_eq_m_times_m(t2, e, t1);
    m_eq_r_times_m(e, R(-0.5), t2);
    for (int k = 0; k < NC * NC; k++) x.e[k] = Cx<R>{radd(x.e[k].re, e.e[k].re), radd(x.e[k].im, e.e[k].im)};
    enorm = fnorm2(e);
  } while (nit < 20 && enorm > eps);
}

template <typename R, int NC>
__device__ void invsqrt_newton(Mat<R, NC>& r, const Mat<R, NC>& a) {
  double ds = fnorm2(a);
  if (ds == 0.0) {
    m_eq_d(r, R(INFINITY));
    return;
  }
  ds = __dsqrt_rn(ds);
  Mat<R, NC> x, e, xi;
  m_eq_d(x, R(1));
  inverse_any(xi, a);
  m_eq_d(e, R(-0.5));
  m_peq_r_times_m(e, (R)__dmul_rn(0.5, ds), xi);
  for (int k = 0; k < NC * NC; k++) x.e[k] = Cx<R>{radd(x.e[k].re, e.e[k].re), radd(x.e[k].im, e.e[k].im)};
  newton_loop(x, e);
  m_eq_r_times_m(r, (R)__ddiv_rn(1.0, __dsqrt_rn(ds)), x);
}

__device__ __constant__ const double kLogP[6] = {7.70838733755885391666E0, 1.79368678507819816313E1,
                                                 1.44989225341610930846E1, 4.70579119878881725854E0,
                                                 4.97494994976747001425E-1, 1.01875663804580931796E-4};
__device__ __constant__ const double kLogQ[5] = {2.31251620126765340583E1, 7.11544750618563894466E1,
                                                 8.29875266912776603211E1, 4.52279145837532221105E1,
                                                 1.12873587189167450590E1};

template <typename R, int NC>
__device__ void log_generic(Mat<R, NC>& r, const Mat<R, NC>& a) {
  double ds = __dsqrt_rn(fnorm2(a));
  if (ds == 0.0) {
    m_eq_d(r, R(-INFINITY));
    return;
  }
  Mat<R, NC> as, as2, as3, t, pa, qa;
  m_eq_r_times_m(as, (R)__ddiv_rn(1.0, ds), a);
  for (int i = 0; i < 4; i++) {
    as2 = as;
    sqrt_newton(as, as2);
  }
  for (int i = 0; i < NC; i++) as(i, i).re = rsub(as(i, i).re, R(1));
  m_eq_d(pa, (R)kLogP[0]);
  m_eq_d(qa, (R)kLogQ[0]);
  m_peq_r_times_m(pa, (R)kLogP[1], as);
  m_peq_r_times_m(qa, (R)kLogQ[1], as);
  m_eq_m_times_m(as2, as, as);
  m_peq_r_times_m(pa, (R)kLogP[2], as2);
  m_peq_r_times_m(qa, (R)kLogQ[2], as2);
  m_eq_m_times_m(as3, as, as2);
  m_peq_r_times_m(pa, (R)kLogP[3], as3);
  m_peq_r_times_m(qa, (R)kLogQ[3], as3);
  m_eq_m_times_m(t, as2, as2);  // as4
  m_peq_r_times_m(pa, (R)kLogP[4], t);
  m_peq_r_times_m(qa, (R)kLogQ[4], t);
  {
    Mat<R, NC> as5;
    m_eq_m_times_m(as5, as, t);
    m_peq_r_times_m(pa, (R)kLogP[5], as5);
    for (int k = 0; k < NC * NC; k++)
      qa.e[k] = Cx<R>{radd(qa.e[k].re, as5.e[k].re), radd(qa.e[k].im, as5.e[k].im)};
  }
  inverse_any(t, qa);  // as5 = qa^-1
  m_eq_m_times_m(qa, pa, t);
  m_eq_m_times_m(pa, as3, qa);
  m_peq_r_times_m(pa, R(-0.5), as2);
  for (int k = 0; k < NC * NC; k++) pa.e[k] = Cx<R>{radd(pa.e[k].re, as.e[k].re), radd(pa.e[k].im, as.e[k].im)};
  m_eq_r_times_m(r, R(16), pa);
  ds = log(ds);
  for (int i = 0; i < NC; i++) r(i, i).re = (R)__dadd_rn((double)r(i, i).re, ds);
}

// ---- eigenvalues by Hessenberg reduction + implicit double-shift QR
// Mixed-precision expressions of the float build (a double literal or
// sqrt() of a float) are evaluated in double and rounded once, as C does.
template <typename R>
__device__ __forceinline__ R rsqrt_c(R x) {
  if constexpr (sizeof(R) == 4) return __fsqrt_rn(x); else return __dsqrt_rn(x);
}
template <typename R>
__device__ __forceinline__ R cabs_q(Cx<R> z) { return rsqrt_c<R>(cnorm2(z)); }
template <typename R>
__device__ __forceinline__ R to_r(double v) {
  if constexpr (sizeof(R) == 4) return __double2float_rn(v); else return v;
}
// QLA_c_eq_c_div_c: t = 1.0/|b|^2 (double division, rounded), then products
template <typename R>
__device__ __forceinline__ Cx<R> cdiv_q(Cx<R> a, Cx<R> b) {
  const R t = to_r<R>(__ddiv_rn(1.0, (double)cnorm2(b)));
  return Cx<R>{rmul(radd(rmul(a.re, b.re), rmul(a.im, b.im)), t), rmul(rsub(rmul(a.im, b.re), rmul(a.re, b.im)), t)};
}
// Hermitian 2x2 eigenvalues (V_eq_eigenvalsH_M.c:82-104)
template <typename R>
__device__ __forceinline__ void eig2_h(Cx<R>& v0, Cx<R>& v1, Cx<R> m00, Cx<R> m01, Cx<R> m10, Cx<R> m11) {
  R det = rsub(rmul(m00.re, m11.re), rmul(m00.im, m11.im));
  det = rsub(det, rsub(rmul(m01.re, m10.re), rmul(m01.im, m10.im)));
  const R tr = radd(m00.re, m11.re);
  if (det == R(0)) {
    v0 = Cx<R>{R(0), R(0)};
    v1 = Cx<R>{tr, R(0)};
  } else {
    const R ss = to_r<R>(__dmul_rn(0.5, (double)tr));
    const R d = rsub(rmul(ss, ss), det);
    const R sd = rsqrt_c<R>(fabs(d));
    const R l1 = radd(ss, copysign(sd, ss));
    v0 = Cx<R>{rdiv(det, l1), R(0)};
    v1 = Cx<R>{l1, R(0)};
  }
}
// general 2x2 eigenvalues (V_eq_eigenvals_M.c:98-124) with QLA's csqrt
template <typename R>
__device__ __forceinline__ void eig2_g(Cx<R>& v0, Cx<R>& v1, Cx<R> m00, Cx<R> m01, Cx<R> m10, Cx<R> m11) {
  Cx<R> det = cmul(m00, m11);
  cmms(det, m01, m10);
  const Cx<R> tr{radd(m00.re, m11.re), radd(m00.im, m11.im)};
  if (det.re == R(0) && det.im == R(0)) {
    v0 = Cx<R>{R(0), R(0)};
    v1 = tr;
  } else {
    const Cx<R> ss{to_r<R>(__dmul_rn(0.5, (double)tr.re)), to_r<R>(__dmul_rn(0.5, (double)tr.im))};
    Cx<R> d = cmul(ss, ss);
    d = Cx<R>{rsub(d.re, det.re), rsub(d.im, det.im)};
    const R nrm = rsqrt_c<R>(cnorm2(d));  // QLA csqrt (lib/cmath/QLA_csqrt.c)
    const R sr = rsqrt_c<R>(fabs(to_r<R>(__dmul_rn(0.5, (double)radd(nrm, d.re)))));
    const R si = copysign(rsqrt_c<R>(fabs(to_r<R>(__dmul_rn(0.5, (double)rsub(nrm, d.re))))), d.im);
    const R ts = radd(rmul(ss.re, sr), rmul(ss.im, si));
    if (ts >= R(0))
      v1 = Cx<R>{radd(ss.re, sr), radd(ss.im, si)};
    else
      v1 = Cx<R>{rsub(ss.re, sr), rsub(ss.im, si)};
    v0 = cdiv_q(det, v1);
  }
}

template <typename R, int NC, bool HERM>
__device__ void eig_qr(Cx<R> (&v)[NC], const Mat<R, NC>& a) {
  Cx<R> mm[NC * NC], h[NC * NC];
  int rc[NC];
  for (int k = 0; k < NC * NC; k++) mm[k] = a.e[k];
  for (int i = 0; i < NC; i++) rc[i] = i;
#define QLAB_MP(i, j) mm[rc[i] * NC + rc[j]]
  for (int k = 0; k < NC - 2; k++) {
    R rmax = cnorm2(QLAB_MP(k + 1, k));
    int imax = k + 1;
    for (int i = k + 2; i < NC; i++) {
      const R n2 = cnorm2(QLAB_MP(i, k));
      if (n2 > rmax) {
        rmax = n2;
        imax = i;
      }
    }
    if (rmax == R(0)) continue;
    {
      const int rk = rc[k + 1];
      rc[k + 1] = rc[imax];
      rc[imax] = rk;
    }
    rmax = rdiv(R(1), rmax);
    const Cx<R> sk{rmul(rmax, QLAB_MP(k + 1, k).re), -rmul(rmax, QLAB_MP(k + 1, k).im)};
    for (int i = k + 2; i < NC; i++) {
      const Cx<R> t = cmul(sk, QLAB_MP(i, k));
      QLAB_MP(i, k) = Cx<R>{R(0), R(0)};
      for (int j = k + 1; j < NC; j++) cmms(QLAB_MP(i, j), t, QLAB_MP(k + 1, j));
      for (int j = 0; j < NC; j++) cpms(QLAB_MP(j, k + 1), t, QLAB_MP(j, i));
    }
  }
  for (int i = 0; i < NC; i++)
    for (int j = 0; j < NC; j++) h[i * NC + j] = QLAB_MP(i, j);
#undef QLAB_MP
#define QLAB_H(i, j) h[(i) * NC + (j)]
  R anorm = R(0);
  for (int i = 0; i < NC; i++)
    for (int j = (i == 0 ? 0 : i - 1); j < NC; j++) anorm = radd(anorm, cabs_q(QLAB_H(i, j)));
  int nn = NC - 1, restarts = 0;
  Cx<R> t{R(0), R(0)};
  while (nn >= 0) {
    int l, its = 0;
    do {
      for (l = nn; l > 0; l--) {
        R s = radd(cabs_q(QLAB_H(l - 1, l - 1)), cabs_q(QLAB_H(l, l)));
        if (s == R(0)) s = anorm;
        const R o = cabs_q(QLAB_H(l, l - 1));
        if (radd(s, o) == s) {
          QLAB_H(l, l - 1) = Cx<R>{R(0), R(0)};
          break;
        }
      }
      Cx<R> x = QLAB_H(nn, nn);
      if (l == nn) {
        v[nn] = Cx<R>{radd(x.re, t.re), radd(x.im, t.im)};
        nn--;
      } else if (l == nn - 1) {
        if constexpr (HERM)
          eig2_h(v[nn - 1], v[nn], QLAB_H(nn - 1, nn - 1), QLAB_H(nn - 1, nn), QLAB_H(nn, nn - 1), x);
        else
          eig2_g(v[nn - 1], v[nn], QLAB_H(nn - 1, nn - 1), QLAB_H(nn - 1, nn), QLAB_H(nn, nn - 1), x);
        v[nn - 1] = Cx<R>{radd(v[nn - 1].re, t.re), radd(v[nn - 1].im, t.im)};
        v[nn] = Cx<R>{radd(v[nn].re, t.re), radd(v[nn].im, t.im)};
        nn -= 2;
      } else {
        if (its >= 100) {
          for (int i = 0; i <= nn; i++) v[i] = Cx<R>{radd(QLAB_H(i, i).re, t.re), radd(QLAB_H(i, i).im, t.im)};
          break;
        }
        Cx<R> y = QLAB_H(nn - 1, nn - 1);
        Cx<R> w = cmul(QLAB_H(nn, nn - 1), QLAB_H(nn - 1, nn));
        if (its == 10 || its == 20) {  // exceptional shift
          t = Cx<R>{radd(t.re, x.re), radd(t.im, x.im)};
          for (int i = 0; i < nn; i++) QLAB_H(i, i) = Cx<R>{rsub(QLAB_H(i, i).re, x.re), rsub(QLAB_H(i, i).im, x.im)};
          QLAB_H(nn, nn) = Cx<R>{R(0), R(0)};
          const R s = radd(cabs_q(QLAB_H(nn, nn - 1)), cabs_q(QLAB_H(nn - 1, nn - 2)));
          x = Cx<R>{to_r<R>(__dmul_rn(0.75, (double)s)), R(0)};
          y = x;
          w = Cx<R>{to_r<R>(__dmul_rn(__dmul_rn(-0.4375, (double)s), (double)s)), R(0)};
        }
        its++;
        const int m = l;
        Cx<R> p, q, r;
        {
          const Cx<R> z = QLAB_H(m, m);
          const Cx<R> rr{rsub(x.re, z.re), rsub(x.im, z.im)};
          const Cx<R> ss{rsub(y.re, z.re), rsub(y.im, z.im)};
          p = cmul(rr, ss);
          p = Cx<R>{rsub(p.re, w.re), rsub(p.im, w.im)};
          cpms(p, QLAB_H(m + 1, m), QLAB_H(m, m + 1));
          Cx<R> t1{rsub(QLAB_H(m + 1, m + 1).re, z.re), rsub(QLAB_H(m + 1, m + 1).im, z.im)};
          t1 = Cx<R>{rsub(t1.re, radd(rr.re, ss.re)), rsub(t1.im, radd(rr.im, ss.im))};
          q = cmul(QLAB_H(m + 1, m), t1);
          r = cmul(QLAB_H(m + 1, m), QLAB_H(m + 2, m + 1));
        }
        for (int k = m; k < nn; k++) {
          R xx = R(0);
          if (k != m) {
            p = QLAB_H(k, k - 1);
            q = QLAB_H(k + 1, k - 1);
            r = Cx<R>{R(0), R(0)};
            if (k + 1 != nn) r = QLAB_H(k + 2, k - 1);
            xx = radd(radd(cabs_q(p), cabs_q(q)), cabs_q(r));
            if (xx != R(0)) {
              const R xxi = rdiv(R(1), xx);
              p = Cx<R>{rmul(xxi, p.re), rmul(xxi, p.im)};
              q = Cx<R>{rmul(xxi, q.re), rmul(xxi, q.im)};
              r = Cx<R>{rmul(xxi, r.re), rmul(xxi, r.im)};
            }
          }
          const R p2 = cnorm2(p);
          const R s2 = radd(radd(p2, cnorm2(q)), cnorm2(r));
          if (s2 != R(0)) {
            Cx<R> sv;
            if (p2 > R(0)) {
              const double sq = __dsqrt_rn((double)rdiv(s2, p2));
              sv = Cx<R>{to_r<R>(__dmul_rn(sq, (double)p.re)), to_r<R>(__dmul_rn(sq, (double)p.im))};
            } else {
              sv = Cx<R>{to_r<R>(__dsqrt_rn((double)s2)), R(0)};
            }
            if (k == m) {
              if (l != m) QLAB_H(k, k - 1) = Cx<R>{-QLAB_H(k, k - 1).re, -QLAB_H(k, k - 1).im};
            } else {
              QLAB_H(k, k - 1) = Cx<R>{rmul(-xx, sv.re), rmul(-xx, sv.im)};
              QLAB_H(k + 1, k - 1) = Cx<R>{R(0), R(0)};
              if (k + 2 < NC) QLAB_H(k + 2, k - 1) = Cx<R>{R(0), R(0)};
            }
            p = Cx<R>{radd(p.re, sv.re), radd(p.im, sv.im)};
            x = cdiv_q(p, sv);
            y = cdiv_q(q, sv);
            w = cdiv_q(r, sv);
            q = cdiv_q(q, p);
            r = cdiv_q(r, p);
            for (int j = k; j <= nn; j++) {  // row modification
              p = QLAB_H(k, j);
              const Cx<R> h1 = QLAB_H(k + 1, j);
              p = Cx<R>{radd(p.re, radd(rmul(q.re, h1.re), rmul(q.im, h1.im))),
                        radd(p.im, rsub(rmul(q.re, h1.im), rmul(q.im, h1.re)))};
              if (k + 1 != nn) {
                const Cx<R> h2 = QLAB_H(k + 2, j);
                p = Cx<R>{radd(p.re, radd(rmul(r.re, h2.re), rmul(r.im, h2.im))),
                          radd(p.im, rsub(rmul(r.re, h2.im), rmul(r.im, h2.re)))};
                cmms(QLAB_H(k + 2, j), p, w);
              }
              cmms(QLAB_H(k + 1, j), p, y);
              cmms(QLAB_H(k, j), p, x);
            }
            const int ie = nn < k + 3 ? nn : k + 3;
            for (int i = l; i <= ie; i++) {  // column modification
              p = cmul(x, QLAB_H(i, k));
              cpms(p, y, QLAB_H(i, k + 1));
              if (k + 1 != nn) {
                cpms(p, w, QLAB_H(i, k + 2));
                Cx<R>& c2 = QLAB_H(i, k + 2);
                c2 = Cx<R>{rsub(c2.re, radd(rmul(p.re, r.re), rmul(p.im, r.im))),
                           rsub(c2.im, rsub(rmul(p.im, r.re), rmul(p.re, r.im)))};
              }
              Cx<R>& c1 = QLAB_H(i, k + 1);
              c1 = Cx<R>{rsub(c1.re, radd(rmul(p.re, q.re), rmul(p.im, q.im))),
                         rsub(c1.im, rsub(rmul(p.im, q.re), rmul(p.re, q.im)))};
              QLAB_H(i, k) = Cx<R>{rsub(QLAB_H(i, k).re, p.re), rsub(QLAB_H(i, k).im, p.im)};
            }
          }
        }
      }
    } while (l + 1 < nn);
    // the template restarts the search without limit; stop after 20 restarts
    if (its >= 100 && ++restarts >= 20) break;
  }
#undef QLAB_H
}

}  // namespace gen

// --------------------------------------------------------------- engine OPs
template <typename R_, int NC, int NB>
struct GenMInverseOp {
  using R = R_;
  static constexpr int NIN = 2, N0 = NC * NC, N1 = NC * NB, N2 = 0, NOUT = NC * NB, NACC = 0;
  __device__ static void apply(const SiteParams& p, const Cx<R> (&a)[N0], const Cx<R> (&b)[N1],
                               const Cx<R> (&d2)[1], Cx<R> (&x)[NOUT]) {
    if constexpr (NC == 3 && NB == 1) {
      MInverseOp<R, 1>::apply(p, a, b, d2, x);
    } else {
      gen::Mat<R, NC> A;
      for (int k = 0; k < N0; k++) A.e[k] = a[k];
      gen::solve_nb<R, NC, NB>(x, A, b);
    }
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[N0], const Cx<R> (&)[N1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

// WHICH: 0 invsqrt, 1 log, 2 expA / expTA at NC != 3 (the exp path),
// 3 sqrtPH at NC != 3 (the sqrt path), 4 invsqrtPH at NC != 3 (invsqrt path)
template <typename R_, int NC, int WHICH>
struct GenMfuncExtOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = NC * NC, N1 = 0, N2 = 0, NOUT = NC * NC, NACC = 0;
  __device__ static void apply(const SiteParams&, const Cx<R> (&a)[N0], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               Cx<R> (&r)[NOUT]) {
    gen::Mat<R, NC> A, X;
    for (int k = 0; k < N0; k++) A.e[k] = a[k];
    if constexpr (WHICH == 0 || WHICH == 4)
      gen::invsqrt_newton(X, A);
    else if constexpr (WHICH == 1)
      gen::log_generic(X, A);
    else if constexpr (WHICH == 2)
      gen::exp_pade(X, A);
    else
      gen::sqrt_newton(X, A);
    for (int k = 0; k < N0; k++) r[k] = X.e[k];
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[N0], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

// eigenvalues at NC != 3 (HERM: eigenvalsH, whose 2x2 step assumes a
// Hermitian block)
template <typename R_, int NC, bool HERM>
struct GenEigenOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = NC * NC, N1 = 0, N2 = 0, NOUT = NC, NACC = 0;
  __device__ static void apply(const SiteParams&, const Cx<R> (&a)[N0], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               Cx<R> (&r)[NOUT]) {
    gen::Mat<R, NC> A;
    for (int k = 0; k < N0; k++) A.e[k] = a[k];
    gen::eig_qr<R, NC, HERM>(r, A);
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[N0], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

}  // namespace qlab
