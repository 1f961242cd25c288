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

}  // namespace qlab
