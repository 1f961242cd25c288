// qla_mfunc.cuh -- colour-matrix functions for Nc = 3 as engine OPs
// (QLA_F3/D3 M_veq_exp_M, M_veq_sqrt_M, M_veq_inverse_M, C_veq_det_M).
//
//  det, inverse: the reference's closed cofactor forms
//    (lib/perl/code-templates/C_eq_det_M.c:70-84, M_eq_inverse_M.c:79-119),
//    restated with explicitly rounded operations in the site precision:
//    bit-identical to the reference for F3 and D3.
//  sqrt: the reference's Newton iteration (M_eq_sqrt_M.c:139-180, with the
//    Gauss-Jordan solve of M_eq_M_inverse_M.c:108-135) in the site precision,
//    the template's own arithmetic (matrices in float for F3, |a|_F and the
//    stopping norm in double, FLT_EPSILON / DBL_EPSILON threshold):
//    bit-identical to QLA_F3 and QLA_D3.
//  exp: Cayley-Hamilton-reduced Taylor series with FP64 coefficients.  With
//    B = A / 2^k (|B|_F <= 1) and B^3 = c2 B^2 + c1 B + c0 1, every power
//    B^j / j! = q0 1 + q1 B + q2 B^2 where (q0,q1,q2) follow the recurrence
//    q' = (q2 c0, q0 + q2 c1, q1 + q2 c2) / (j+1); summing the terms gives
//    exp(B) = f0 1 + f1 B + f2 B^2 with no eigenvalues involved, so nearly
//    degenerate spectra need no special case; then k squarings.  D3: all of
//    it in FP64 (26 terms).  F3: only the coefficients in FP64 (16 terms);
//    B^2, the assembly and the squarings in FP32.  The reference's F3/D3 use a
//    rational approximation with scaling (M_eq_exp_M.c:302-367); agreement is
//    checked against its FP64 (D3) result.
#pragma once
#include "qla_engine.cuh"

namespace qlab {

template <typename R>
using C9 = Cx<R>[9];

__device__ __forceinline__ Cx<double> cd(Cx<float> v) { return Cx<double>{(double)v.re, (double)v.im}; }
__device__ __forceinline__ Cx<double> cd(Cx<double> v) { return v; }
template <typename R>
__device__ __forceinline__ Cx<R> cround(Cx<double> v) {
  return Cx<R>{(R)v.re, (R)v.im};
}

// explicitly rounded complex helpers (qla_complex.h order)
template <typename R>
__device__ __forceinline__ Cx<R> cmul(Cx<R> a, Cx<R> b) {  // c_eq_c_times_c
  return Cx<R>{rsub(rmul(a.re, b.re), rmul(a.im, b.im)), radd(rmul(a.re, b.im), rmul(a.im, b.re))};
}
template <typename R>
__device__ __forceinline__ void cmms(Cx<R>& c, Cx<R> a, Cx<R> b) {  // c_meq_c_times_c
  c.re = rsub(c.re, rsub(rmul(a.re, b.re), rmul(a.im, b.im)));
  c.im = rsub(c.im, radd(rmul(a.re, b.im), rmul(a.im, b.re)));
}
template <typename R>
__device__ __forceinline__ void cpms(Cx<R>& c, Cx<R> a, Cx<R> b) {  // c_peq_c_times_c
  c.re = radd(c.re, rsub(rmul(a.re, b.re), rmul(a.im, b.im)));
  c.im = radd(c.im, radd(rmul(a.re, b.im), rmul(a.im, b.re)));
}
template <typename R>
__device__ __forceinline__ R cnorm2(Cx<R> a) {
  return radd(rmul(a.re, a.re), rmul(a.im, a.im));
}

// r = a * b for 3x3 (M_eq_M_times_M order: x = 0; x += a_ik b_kj)
template <typename R>
__device__ __forceinline__ void mat3_mul(Cx<R> (&r)[9], const Cx<R> (&a)[9], const Cx<R> (&b)[9]) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      Cx<R> x{R(0), R(0)};
#pragma unroll
      for (int k = 0; k < 3; k++) cpms(x, a[i * 3 + k], b[k * 3 + j]);
      r[i * 3 + j] = x;
    }
}

// sum |a_ij|^2, each term in R, summed in double (the templates' maxev2)
template <typename R>
__device__ __forceinline__ double fnorm2_3(const Cx<R> (&a)[9]) {
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 9; k++) s = __dadd_rn(s, (double)cnorm2(a[k]));
  return s;
}

// ---------------------------------------------------------------------------
// C_eq_det_M (nc = 3)
template <typename R>
__device__ __forceinline__ Cx<R> det3(const Cx<R> (&a)[9]) {
  Cx<R> det2 = cmul(a[0], a[4]);
  cmms(det2, a[1], a[3]);
  Cx<R> det1 = cmul(a[2], a[3]);
  cmms(det1, a[0], a[5]);
  Cx<R> det0 = cmul(a[1], a[5]);
  cmms(det0, a[2], a[4]);
  Cx<R> det = cmul(det2, a[8]);
  cpms(det, det1, a[7]);
  cpms(det, det0, a[6]);
  return det;
}

template <typename R_>
struct DetOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = 9, N1 = 0, N2 = 0, NOUT = 1, NACC = 0;
  __device__ __forceinline__ static void apply(const SiteParams&, const Cx<R> (&a)[9], const Cx<R> (&)[1],
                                               const Cx<R> (&)[1], Cx<R> (&y)[1]) {
    y[0] = det3(a);
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[9], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

// ---------------------------------------------------------------------------
// M_eq_inverse_M (nc = 3): cofactors times 1/det
template <typename R>
__device__ __forceinline__ void inv3(Cx<R> (&x)[9], const Cx<R> (&a)[9]) {
  Cx<R> det2 = cmul(a[0], a[4]);
  cmms(det2, a[1], a[3]);
  Cx<R> det1 = cmul(a[2], a[3]);
  cmms(det1, a[0], a[5]);
  Cx<R> det0 = cmul(a[1], a[5]);
  cmms(det0, a[2], a[4]);
  Cx<R> det = cmul(det2, a[8]);
  cpms(det, det1, a[7]);
  cpms(det, det0, a[6]);
  // QLA_c_eq_r_div_c(idet, 1, det): t = 1/|det|^2; idet = t*conj(det)
  const R t = rdiv(R(1), cnorm2(det));
  const Cx<R> idet{rmul(t, det.re), rmul(-t, det.im)};
#define QLAB_SET(i0, j0, i1, j1, i2, j2)              \
  {                                                   \
    Cx<R> d_ = cmul(a[i1 * 3 + j1], a[i2 * 3 + j2]);  \
    cmms(d_, a[i1 * 3 + j2], a[i2 * 3 + j1]);         \
    x[i0 * 3 + j0] = cmul(d_, idet);                  \
  }
  QLAB_SET(0, 0, 1, 1, 2, 2);
  QLAB_SET(0, 1, 2, 1, 0, 2);
  x[2] = cmul(det0, idet);
  QLAB_SET(1, 0, 1, 2, 2, 0);
  QLAB_SET(1, 1, 2, 2, 0, 0);
  x[5] = cmul(det1, idet);
  QLAB_SET(2, 0, 1, 0, 2, 1);
  QLAB_SET(2, 1, 2, 0, 0, 1);
  x[8] = cmul(det2, idet);
#undef QLAB_SET
}

template <typename R_>
struct InverseOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = 9, N1 = 0, N2 = 0, NOUT = 9, NACC = 0;
  __device__ __forceinline__ static void apply(const SiteParams&, const Cx<R> (&a)[9], const Cx<R> (&)[1],
                                               const Cx<R> (&)[1], Cx<R> (&x)[9]) {
    inv3(x, a);
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[9], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

// ---------------------------------------------------------------------------
// x = a^-1 b, Gauss-Jordan with partial pivoting (M_eq_M_inverse_M.c:108-135)
// for NB right-hand-side columns, rows swapped physically (same arithmetic
// as the template's row permutation).  Result written into d (in place of
// the right-hand side).
template <typename R, int NB = 3>
__device__ __forceinline__ void gj_solve3(Cx<R> (&c)[9], Cx<R> (&d)[3 * NB]) {
#pragma unroll
  for (int k = 0; k < 3; k++) {
    R rmax = cnorm2(c[k * 3 + k]);
    int imax = k;
#pragma unroll
    for (int i = k + 1; i < 3; i++) {
      const R rr = cnorm2(c[i * 3 + k]);
      if (rr > rmax) {
        rmax = rr;
        imax = i;
      }
    }
#pragma unroll
    for (int i = k + 1; i < 3; i++) {
      if (imax == i) {
#pragma unroll
        for (int j = 0; j < 3; j++) {
          const Cx<R> t = c[k * 3 + j];
          c[k * 3 + j] = c[i * 3 + j];
          c[i * 3 + j] = t;
        }
#pragma unroll
        for (int j = 0; j < NB; j++) {
          const Cx<R> t = d[k * NB + j];
          d[k * NB + j] = d[i * NB + j];
          d[i * NB + j] = t;
        }
      }
    }
    rmax = rdiv(R(1), rmax);
    const Cx<R> s{rmul(rmax, c[k * 3 + k].re), -rmul(rmax, c[k * 3 + k].im)};
    c[k * 3 + k] = s;
#pragma unroll
    for (int i = 0; i < 3; i++) {
      if (i == k) continue;
      const Cx<R> t = cmul(s, c[i * 3 + k]);
#pragma unroll
      for (int j = k + 1; j < 3; j++) cmms(c[i * 3 + j], t, c[k * 3 + j]);
#pragma unroll
      for (int j = 0; j < NB; j++) cmms(d[i * NB + j], t, d[k * NB + j]);
    }
  }
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < NB; j++) d[i * NB + j] = cmul(c[i * 3 + i], d[i * NB + j]);
}

// Newton loop of M_eq_sqrt_M.c:158-171 / M_eq_invsqrt_M.c:160-173 in the
// site precision R, the templates' own arithmetic (QLA_F3 in float, QLA_D3 in
// double): e <- -1/2 e x^-1 e, x += e until |e|_F^2 <= EPS (FLT_EPSILON or
// DBL_EPSILON; the norm's terms in R, summed in double) or 20 iterations.
template <typename R>
__device__ __forceinline__ void newton_sqrt3(Cx<R> (&x)[9], Cx<R> (&e)[9]) {
  const double eps = sizeof(R) == 4 ? 1.1920928955078125e-07 : 2.220446049250313080847e-16;
  Cx<R> c[9], d[9];
  int nit = 0;
  double enorm;
  do {
    nit++;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      c[k] = x[k];
      d[k] = e[k];
    }
    gj_solve3(c, d);    // d = x^-1 e
    mat3_mul(c, e, d);  // c = e x^-1 e
#pragma unroll
    for (int k = 0; k < 9; k++) {
      e[k] = Cx<R>{rmul(R(-0.5), c[k].re), rmul(R(-0.5), c[k].im)};
      x[k] = Cx<R>{radd(x[k].re, e[k].re), radd(x[k].im, e[k].im)};
    }
    enorm = fnorm2_3(e);
  } while (nit < 20 && enorm > eps);
}

// M_eq_sqrt_M in the site precision R: r = sqrt(a).  ds = |a|_F is formed in
// double and enters as (R)(1/ds) and (R)sqrt(ds), as the template's
// M_eq_d_times_M does (QLA_Real rr = d).
template <typename R>
__device__ __forceinline__ void sqrt3(Cx<R> (&r)[9], const Cx<R> (&a)[9]) {
  double ds = fnorm2_3(a);
  if (ds == 0.0) {
#pragma unroll
    for (int k = 0; k < 9; k++) r[k] = Cx<R>{R(0), R(0)};
    return;
  }
  ds = __dsqrt_rn(ds);
  Cx<R> x[9], e[9];
  const R inv = (R)__ddiv_rn(1.0, ds);
#pragma unroll
  for (int k = 0; k < 9; k++) {
    x[k] = Cx<R>{rmul(inv, a[k].re), rmul(inv, a[k].im)};  // x = a / ds
    const R dg = (k % 4 == 0) ? R(0.5) : R(0);               // e = 0.5 1 - 0.5 x
    e[k] = Cx<R>{radd(dg, rmul(R(-0.5), x[k].re)), radd(R(0), rmul(R(-0.5), x[k].im))};
    x[k] = Cx<R>{radd(x[k].re, e[k].re), radd(x[k].im, e[k].im)};
  }
  newton_sqrt3(x, e);
  const R sds = (R)__dsqrt_rn(ds);
#pragma unroll
  for (int k = 0; k < 9; k++) r[k] = Cx<R>{rmul(sds, x[k].re), rmul(sds, x[k].im)};
}

// M_eq_sqrt_M (Newton) in the site precision: bit-identical to QLA_F3 / QLA_D3
template <typename R_>
struct SqrtOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = 9, N1 = 0, N2 = 0, NOUT = 9, NACC = 0;
  __device__ static void apply(const SiteParams&, const Cx<R> (&a)[9], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               Cx<R> (&r)[9]) {
    sqrt3(r, a);
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[9], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

// plain complex arithmetic (the compiler may fuse multiply-adds): for the
// F3 exp, whose result is not tied to the reference's rounding sequence
template <typename T>
__device__ __forceinline__ Cx<T> cmul_fast(Cx<T> a, Cx<T> b) {
  return Cx<T>{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename T>
__device__ __forceinline__ void mat3_mul_fast(Cx<T> (&r)[9], const Cx<T> (&a)[9], const Cx<T> (&b)[9]) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      Cx<T> x = cmul_fast(a[i * 3], b[j]);
#pragma unroll
      for (int k = 1; k < 3; k++) {
        const Cx<T> t = cmul_fast(a[i * 3 + k], b[k * 3 + j]);
        x.re += t.re;
        x.im += t.im;
      }
      r[i * 3 + j] = x;
    }
}
template <typename T>
__device__ __forceinline__ Cx<T> det3_fast(const Cx<T> (&a)[9]) {
  Cx<T> m0 = cmul_fast(a[4], a[8]), m1 = cmul_fast(a[5], a[7]);
  Cx<T> n0 = cmul_fast(a[3], a[8]), n1 = cmul_fast(a[5], a[6]);
  Cx<T> o0 = cmul_fast(a[3], a[7]), o1 = cmul_fast(a[4], a[6]);
  const Cx<T> c0{m0.re - m1.re, m0.im - m1.im}, c1{n0.re - n1.re, n0.im - n1.im}, c2{o0.re - o1.re, o0.im - o1.im};
  const Cx<T> t0 = cmul_fast(a[0], c0), t1 = cmul_fast(a[1], c1), t2 = cmul_fast(a[2], c2);
  return Cx<T>{t0.re - t1.re + t2.re, t0.im - t1.im + t2.im};
}

// ---------------------------------------------------------------------------
// M_eq_exp_M: Cayley-Hamilton-reduced Taylor series (see header)
template <typename R_>
struct ExpOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = 9, N1 = 0, N2 = 0, NOUT = 9, NACC = 0;
  static constexpr int kTerms = 26;
  // F3: 16 terms (the neglected tail is below 1/17! < 3e-15 of the result's
  // scale when |B|_F <= 1)
  static constexpr int kTermsF3 = 16;
  __device__ static void apply(const SiteParams& p, const Cx<R> (&a)[9], const Cx<R> (&x1)[1],
                               const Cx<R> (&x2)[1], Cx<R> (&r)[9]) {
    if constexpr (sizeof(R) == 4)
      apply_f3(a, r);
    else
      apply_d3(p, a, x1, x2, r);
  }

  // F3: FP64 only for the Cayley-Hamilton coefficients (the traces, the
  // determinant and the Taylor recurrence on q0, q1, q2, computed from the
  // exactly promoted float B); B^2, the assembly f0 + f1 B + f2 B^2 and the
  // squarings in FP32 with fused multiply-adds.
  __device__ static void apply_f3(const Cx<float> (&a)[9], Cx<float> (&r)[9]) {
    double fn = 0.0;
#pragma unroll
    for (int k = 0; k < 9; k++) fn = fma((double)a[k].im, (double)a[k].im, fma((double)a[k].re, (double)a[k].re, fn));
    // B = A / 2^ks with |B|_F^2 <= 1: fn < 2^E, so ks = ceil(E / 2) suffices
    int ks = 0;
    if (fn > 1.0) {
      int E;
      frexp(fn, &E);
      ks = (E + 1) >> 1;
      if (ks > 60) ks = 60;
    }
    const float sc = ldexpf(1.0f, -ks);  // exact power of two
    Cx<float> b[9];
#pragma unroll
    for (int k = 0; k < 9; k++) b[k] = Cx<float>{a[k].re * sc, a[k].im * sc};
    // coefficients in FP64: tr B, tr B^2 = sum_ik b_ik b_ki, det B
    Cx<double> bd[9];
#pragma unroll
    for (int k = 0; k < 9; k++) bd[k] = cd(b[k]);
    const Cx<double> trb{bd[0].re + bd[4].re + bd[8].re, bd[0].im + bd[4].im + bd[8].im};
    Cx<double> trb2{0.0, 0.0};
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const Cx<double> u = bd[i * 3 + k], v = bd[k * 3 + i];
        trb2.re = fma(u.re, v.re, fma(-u.im, v.im, trb2.re));
        trb2.im = fma(u.re, v.im, fma(u.im, v.re, trb2.im));
      }
    const Cx<double> c2 = trb;
    const Cx<double> c1{-0.5 * (trb.re * trb.re - trb.im * trb.im - trb2.re),
                        -0.5 * (2.0 * trb.re * trb.im - trb2.im)};
    const Cx<double> c0 = det3_fast(bd);
    Cx<double> q0{1.0, 0.0}, q1{0.0, 0.0}, q2{0.0, 0.0};
    Cx<double> f0 = q0, f1 = q1, f2 = q2;
#pragma unroll 3
    for (int j = 1; j < kTermsF3; j++) {
      const double inv = 1.0 / (double)j;
      const Cx<double> n0 = cmul_fast(q2, c0);
      Cx<double> n1 = cmul_fast(q2, c1);
      Cx<double> n2 = cmul_fast(q2, c2);
      n1.re += q0.re;
      n1.im += q0.im;
      n2.re += q1.re;
      n2.im += q1.im;
      q0 = Cx<double>{n0.re * inv, n0.im * inv};
      q1 = Cx<double>{n1.re * inv, n1.im * inv};
      q2 = Cx<double>{n2.re * inv, n2.im * inv};
      f0.re += q0.re;
      f0.im += q0.im;
      f1.re += q1.re;
      f1.im += q1.im;
      f2.re += q2.re;
      f2.im += q2.im;
    }
    const Cx<float> g0{(float)f0.re, (float)f0.im}, g1{(float)f1.re, (float)f1.im}, g2{(float)f2.re, (float)f2.im};
    // FP32: B^2, the assembly, the squarings
    Cx<float> b2[9], e[9];
    mat3_mul_fast(b2, b, b);
#pragma unroll
    for (int k = 0; k < 9; k++) {
      Cx<float> t = cmul_fast(g1, b[k]);
      const Cx<float> u = cmul_fast(g2, b2[k]);
      t.re += u.re;
      t.im += u.im;
      if (k % 4 == 0) {
        t.re += g0.re;
        t.im += g0.im;
      }
      e[k] = t;
    }
    for (int s = 0; s < ks; s++) {
      mat3_mul_fast(b2, e, e);
#pragma unroll
      for (int k = 0; k < 9; k++) e[k] = b2[k];
    }
#pragma unroll
    for (int k = 0; k < 9; k++) r[k] = e[k];
  }

  // D3: the whole evaluation in FP64
  __device__ static void apply_d3(const SiteParams&, const Cx<R> (&a)[9], const Cx<R> (&)[1], const Cx<R> (&)[1],
                                  Cx<R> (&r)[9]) {
    Cx<double> b[9];
#pragma unroll
    for (int k = 0; k < 9; k++) b[k] = cd(a[k]);
    double fn = 0.0;
#pragma unroll
    for (int k = 0; k < 9; k++) fn += b[k].re * b[k].re + b[k].im * b[k].im;
    // scale by 2^-k so that |B|_F <= 1 (exact: a power of two)
    int ks = 0;
    if (fn > 1.0) {
      ks = (int)ceil(0.5 * log2(fn));
      if (ks > 60) ks = 60;
      const double sc = ldexp(1.0, -ks);
#pragma unroll
      for (int k = 0; k < 9; k++) b[k] = Cx<double>{b[k].re * sc, b[k].im * sc};
    }
    Cx<double> b2[9];
    mat3_mul(b2, b, b);
    const Cx<double> trb{b[0].re + b[4].re + b[8].re, b[0].im + b[4].im + b[8].im};
    const Cx<double> trb2{b2[0].re + b2[4].re + b2[8].re, b2[0].im + b2[4].im + b2[8].im};
    const Cx<double> trb_sq = cmul(trb, trb);
    // B^3 = c2 B^2 + c1 B + c0 1  (Cayley-Hamilton)
    const Cx<double> c2 = trb;
    const Cx<double> c1{-0.5 * (trb_sq.re - trb2.re), -0.5 * (trb_sq.im - trb2.im)};
    const Cx<double> c0 = det3(b);
    Cx<double> q0{1.0, 0.0}, q1{0.0, 0.0}, q2{0.0, 0.0};
    Cx<double> f0 = q0, f1 = q1, f2 = q2;
#pragma unroll 2
    for (int j = 1; j < kTerms; j++) {
      const double inv = 1.0 / (double)j;
      const Cx<double> n0 = cmul(q2, c0);
      Cx<double> n1 = cmul(q2, c1);
      Cx<double> n2 = cmul(q2, c2);
      n1.re += q0.re;
      n1.im += q0.im;
      n2.re += q1.re;
      n2.im += q1.im;
      q0 = Cx<double>{n0.re * inv, n0.im * inv};
      q1 = Cx<double>{n1.re * inv, n1.im * inv};
      q2 = Cx<double>{n2.re * inv, n2.im * inv};
      f0.re += q0.re;
      f0.im += q0.im;
      f1.re += q1.re;
      f1.im += q1.im;
      f2.re += q2.re;
      f2.im += q2.im;
    }
    Cx<double> e[9];
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const Cx<double> t1 = cmul(f1, b[k]);
      const Cx<double> t2 = cmul(f2, b2[k]);
      e[k] = Cx<double>{t1.re + t2.re, t1.im + t2.im};
      if (k % 4 == 0) {
        e[k].re += f0.re;
        e[k].im += f0.im;
      }
    }
    for (int s = 0; s < ks; s++) {
      mat3_mul(b2, e, e);
#pragma unroll
      for (int k = 0; k < 9; k++) e[k] = b2[k];
    }
#pragma unroll
    for (int k = 0; k < 9; k++) r[k] = cround<R>(e[k]);
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[9], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

}  // namespace qlab
