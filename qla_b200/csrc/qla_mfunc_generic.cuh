// qla_mfunc_generic.cuh -- the reference's generic colour-matrix functions for
// a compile-time colour count NC (QLA_FN_ at nc = NC), as engine OPs.
//
// Restated from lib/perl/code-templates, with every multiply, add and divide
// rounded explicitly in the site precision R and in the templates' order, so
// results are bit-identical to the reference's N-colour build:
//   exp     M_eq_exp_M.c:302-367 (s = ceil(2|A|_F) <= 1024 scaling, rational
//           approximation with P and Q, binary powering);
//   sqrt    M_eq_sqrt_M.c:139-180 (Newton, FLT/DBL_EPSILON, 20 iterations);
//   inverse M_eq_inverse_M.c:79-119 (NC = 3 cofactors) / :120-162 (Gauss-Jordan);
//   det     C_eq_det_M.c:70-84 (NC = 3) / :86-143 (LU with pivoting);
//   x = a^-1 b  M_eq_M_inverse_M.c:108-135 (Gauss-Jordan, used by exp and sqrt).
// The work matrices live in thread-local arrays (registers for small NC, local
// memory for NC = 8); these functions are FP-issue-bound, not HBM-bound.
#pragma once
#include "qla_mfunc.cuh"

namespace qlab {
namespace gen {

template <typename R, int NC>
struct Mat {
  Cx<R> e[NC * NC];
  __device__ __forceinline__ Cx<R>& operator()(int i, int j) { return e[i * NC + j]; }
  __device__ __forceinline__ const Cx<R>& operator()(int i, int j) const { return e[i * NC + j]; }
};

template <typename R, int NC>
__device__ __forceinline__ void m_eq_d(Mat<R, NC>& r, R d) {
#pragma unroll
  for (int i = 0; i < NC; i++)
#pragma unroll
    for (int j = 0; j < NC; j++) r(i, j) = Cx<R>{i == j ? d : R(0), R(0)};
}

template <typename R, int NC>
__device__ __forceinline__ void m_peq_r_times_m(Mat<R, NC>& r, R s, const Mat<R, NC>& a) {
#pragma unroll
  for (int k = 0; k < NC * NC; k++) {
    r.e[k].re = radd(r.e[k].re, rmul(s, a.e[k].re));
    r.e[k].im = radd(r.e[k].im, rmul(s, a.e[k].im));
  }
}

template <typename R, int NC>
__device__ __forceinline__ void m_eq_r_times_m(Mat<R, NC>& r, R s, const Mat<R, NC>& a) {
#pragma unroll
  for (int k = 0; k < NC * NC; k++) r.e[k] = Cx<R>{rmul(s, a.e[k].re), rmul(s, a.e[k].im)};
}

template <typename R, int NC>
__device__ __forceinline__ void m_eq_m_times_m(Mat<R, NC>& r, const Mat<R, NC>& a, const Mat<R, NC>& b) {
  for (int i = 0; i < NC; i++)
    for (int j = 0; j < NC; j++) {
      Cx<R> x{R(0), R(0)};
#pragma unroll
      for (int k = 0; k < NC; k++) cpms(x, a(i, k), b(k, j));
      r(i, j) = x;
    }
}

template <typename R, int NC>
__device__ __forceinline__ double fnorm2(const Mat<R, NC>& a) {
  double s = 0.0;
  for (int k = 0; k < NC * NC; k++) s = __dadd_rn(s, (double)cnorm2(a.e[k]));
  return s;
}

// x = a^-1 b, Gauss-Jordan with partial pivoting through a row permutation
template <typename R, int NC>
__device__ void m_eq_m_inverse_m(Mat<R, NC>& x, const Mat<R, NC>& a, const Mat<R, NC>& b) {
  Mat<R, NC> c = a, d = b;
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
      for (int j = 0; j < NC; j++) cmms(d(ri, j), t, d(rkk, j));
    }
  }
  for (int i = 0; i < NC; i++)
    for (int j = 0; j < NC; j++) x(i, j) = cmul(c(row[i], i), d(row[i], j));
}

__device__ __constant__ const double kPadeP[3] = {9.99999999999999999910E-1, 3.02994407707441961300E-2,
                                                  1.26177193074810590878E-4};
__device__ __constant__ const double kPadeQ[4] = {2.00000000000000000009E0, 2.27265548208155028766E-1,
                                                  2.52448340349684104192E-3, 3.00198505138664455042E-6};

template <typename R, int NC>
__device__ void exp_pade(Mat<R, NC>& r, const Mat<R, NC>& a) {
  double ds = __dsqrt_rn(fnorm2(a));
  if (ds == 0.0) {
    m_eq_d(r, R(1));
    return;
  }
  unsigned s = (unsigned)ceil(__dmul_rn(2.0, ds));
  if (s > 1024u) s = 1024u;
  ds = (double)s;
  Mat<R, NC> bs, bs2, bs4, bs6, pb, qb;
  const R dsi = (R)__ddiv_rn(1.0, ds);
  m_eq_r_times_m(bs, dsi, a);
  m_eq_d(pb, (R)kPadeP[0]);
  m_eq_d(qb, (R)kPadeQ[0]);
  m_eq_m_times_m(bs2, bs, bs);
  m_peq_r_times_m(pb, (R)kPadeP[1], bs2);
  m_peq_r_times_m(qb, (R)kPadeQ[1], bs2);
  m_eq_m_times_m(bs4, bs2, bs2);
  m_peq_r_times_m(pb, (R)kPadeP[2], bs4);
  m_peq_r_times_m(qb, (R)kPadeQ[2], bs4);
  m_eq_m_times_m(bs6, bs4, bs2);
  m_peq_r_times_m(qb, (R)kPadeQ[3], bs6);
  m_eq_m_times_m(bs6, bs, pb);
  for (int k = 0; k < NC * NC; k++) pb.e[k] = Cx<R>{rsub(qb.e[k].re, bs6.e[k].re), rsub(qb.e[k].im, bs6.e[k].im)};
  m_eq_m_inverse_m(qb, pb, bs6);
  m_eq_d(pb, R(1));
  m_peq_r_times_m(pb, R(2), qb);
  if (s == 1u) {
    r = pb;
    return;
  }
  // binary powering: va accumulates, vb squares (the template's pointer swaps
  // become copies)
  Mat<R, NC> va, t;
  m_eq_d(va, R(1));
  for (; s > 0u; s >>= 1) {
    if (s & 1u) {
      m_eq_m_times_m(t, va, pb);
      va = t;
    }
    m_eq_m_times_m(t, pb, pb);
    pb = t;
  }
  r = va;
}

template <typename R, int NC>
__device__ void sqrt_newton(Mat<R, NC>& r, const Mat<R, NC>& a) {
  double ds = fnorm2(a);
  if (ds == 0.0) {
    m_eq_d(r, R(0));
    return;
  }
  ds = __dsqrt_rn(ds);
  Mat<R, NC> x, e, t1, t2;
  m_eq_r_times_m(x, (R)__ddiv_rn(1.0, ds), a);
  m_eq_d(e, R(0.5));
  m_peq_r_times_m(e, R(-0.5), x);
  for (int k = 0; k < NC * NC; k++) x.e[k] = Cx<R>{radd(x.e[k].re, e.e[k].re), radd(x.e[k].im, e.e[k].im)};
  const double eps = sizeof(R) == 4 ? 1.1920928955078125e-07 : 2.220446049250313080847e-16;
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
  m_eq_r_times_m(r, (R)__dsqrt_rn(ds), x);
}

template <typename R, int NC>
__device__ Cx<R> det_lu(const Mat<R, NC>& a) {
  Mat<R, NC> c = a;
  int row[NC], nswaps = 0;
#pragma unroll
  for (int i = 0; i < NC; i++) row[i] = i;
  Cx<R> x{R(1), R(0)};
  for (int j = 0; j < NC; j++) {
    if (j > 0) {
      for (int i = j; i < NC; i++) {
        Cx<R> t2 = c(row[i], j);
        for (int k = 0; k < j; k++) cmms(t2, c(row[i], k), c(row[k], j));
        c(row[i], j) = t2;
      }
    }
    R rmax = cnorm2(c(row[j], j));
    int kmax = j;
    for (int k = j + 1; k < NC; k++) {
      const R rr = cnorm2(c(row[k], j));
      if (rr > rmax) {
        rmax = rr;
        kmax = k;
      }
    }
    if (rmax == R(0)) return Cx<R>{R(0), R(0)};
    if (kmax != j) {
      const int rj = row[j];
      row[j] = row[kmax];
      row[kmax] = rj;
      nswaps++;
    }
    x = cmul(x, c(row[j], j));
    const R ri = rdiv(R(1), rmax);
    const Cx<R> cjji{rmul(ri, c(row[j], j).re), -rmul(ri, c(row[j], j).im)};
    for (int i = j + 1; i < NC; i++) {
      Cx<R> t2 = c(row[j], i);
      for (int k = 0; k < j; k++) cmms(t2, c(row[j], k), c(row[k], i));
      c(row[j], i) = cmul(t2, cjji);
    }
  }
  if (nswaps & 1) x = Cx<R>{-x.re, -x.im};
  return x;
}

}  // namespace gen

// --------------------------------------------------------------- engine OPs
template <typename R_, int NC>
struct GenExpOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = NC * NC, N1 = 0, N2 = 0, NOUT = NC * NC, NACC = 0;
  __device__ static void apply(const SiteParams&, const Cx<R> (&a)[N0], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               Cx<R> (&r)[NOUT]) {
    gen::Mat<R, NC> A, X;
    for (int k = 0; k < N0; k++) A.e[k] = a[k];
    gen::exp_pade(X, A);
    for (int k = 0; k < N0; k++) r[k] = X.e[k];
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[N0], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

template <typename R_, int NC>
struct GenSqrtOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = NC * NC, N1 = 0, N2 = 0, NOUT = NC * NC, NACC = 0;
  __device__ static void apply(const SiteParams&, const Cx<R> (&a)[N0], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               Cx<R> (&r)[NOUT]) {
    gen::Mat<R, NC> A, X;
    for (int k = 0; k < N0; k++) A.e[k] = a[k];
    gen::sqrt_newton(X, A);
    for (int k = 0; k < N0; k++) r[k] = X.e[k];
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[N0], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

template <typename R_, int NC>
struct GenInverseOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = NC * NC, N1 = 0, N2 = 0, NOUT = NC * NC, NACC = 0;
  __device__ static void apply(const SiteParams& p, const Cx<R> (&a)[N0], const Cx<R> (&d1)[1],
                               const Cx<R> (&d2)[1], Cx<R> (&r)[NOUT]) {
    if constexpr (NC == 3) {
      InverseOp<R>::apply(p, a, d1, d2, r);
    } else {
      gen::Mat<R, NC> A, I, X;
      for (int k = 0; k < N0; k++) A.e[k] = a[k];
      gen::m_eq_d(I, R(1));
      gen::m_eq_m_inverse_m(X, A, I);
      for (int k = 0; k < N0; k++) r[k] = X.e[k];
    }
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[N0], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

template <typename R_, int NC>
struct GenDetOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = NC * NC, N1 = 0, N2 = 0, NOUT = 1, NACC = 0;
  __device__ static void apply(const SiteParams&, const Cx<R> (&a)[N0], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               Cx<R> (&r)[1]) {
    if constexpr (NC == 3) {
      r[0] = det3(a);
    } else {
      gen::Mat<R, NC> A;
      for (int k = 0; k < N0; k++) A.e[k] = a[k];
      r[0] = gen::det_lu(A);
    }
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[N0], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

}  // namespace qlab
