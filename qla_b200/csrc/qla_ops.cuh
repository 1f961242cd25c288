// qla_ops.cuh -- per-site operators of the level-1 families, as engine OPs.
//
// Each OP restates, for one site, the loop body that the reference generator
// emits for its family; eqop/mu/sign stay runtime-uniform parameters so that
// one kernel serves all eqop variants of a family.
#pragma once
#include "qla_engine.cuh"

namespace qlab {

template <typename R>
using CxArr1 = Cx<R>[1];

// ---------------------------------------------------------------------------
// r (eqop) A * B, A = a | a^+ (colour matrix), B = b (NC x NCOL) | b^+ (matrix).
// Restates lib/perl/build_qla.pl:1588-1622 + expressions_tensor.pl:766: per
// output element x = (peq|meq ? r : 0); x (+|-)= A(i,k) B(k,s) for k in order.
// (the record arrays may be longer than the records: callers that keep
// records of several kinds in one fixed-size array pass that array)
template <typename R, int NC, int NCOL, bool ADJA, bool ADJB, int LA, int LB, int LY>
__device__ __forceinline__ void lmult_site(int eqop, bool load, const Cx<R> (&a)[LA], const Cx<R> (&b)[LB],
                                           Cx<R> (&y)[LY]) {
  static_assert(LA >= NC * NC && LB >= NC * NCOL && LY >= NC * NCOL, "record array too short");
  const bool minus = (eqop == MEQ || eqop == EQM);
#pragma unroll
  for (int ic = 0; ic < NC; ic++) {
#pragma unroll
    for (int s = 0; s < NCOL; s++) {
      Cx<R> x;
      if (load) {
        x = y[ic * NCOL + s];
      } else {
        x.re = R(0);
        x.im = R(0);
      }
#pragma unroll
      for (int kc = 0; kc < NC; kc++) {
        const Cx<R> av = ADJA ? a[kc * NC + ic] : a[ic * NC + kc];
        const Cx<R> bv = ADJB ? b[s * NCOL + kc] : b[kc * NCOL + s];
        cmac<ADJA, ADJB>(x, minus, av, bv);
      }
      y[ic * NCOL + s] = x;
    }
  }
}

template <typename R_, int NC, int NCOL, bool ADJA, bool ADJB>
struct LMultOp {
  using R = R_;
  static constexpr int NIN = 2, N0 = NC * NC, N1 = NC * NCOL, N2 = 0, NOUT = NC * NCOL, NACC = 0;
  __device__ __forceinline__ static void apply(const SiteParams& p, const Cx<R> (&a)[N0], const Cx<R> (&b)[N1],
                                               const Cx<R> (&)[1], Cx<R> (&y)[NOUT]) {
    lmult_site<R, NC, NCOL, ADJA, ADJB>(p.eqop, p.out_read != 0, a, b, y);
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[N0], const Cx<R> (&)[N1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

// ---------------------------------------------------------------------------
// Spin projection / reconstruction.  Gamma basis and component tables restate
// lib/perl/expressions_gamma.pl:59-91 (basis), :244-275 (projection onto a
// HalfFermion) and :309-337 (reconstruction).  Entries: {kind, spin_a, spin_b}
// with kind 0 c+c, 1 c-c, 2 c+ic, 3 c-ic, 4 copy.
// c (eqop) a (+|-) (i) b ; qla_complex.h:147-154, 287-324 (eqm forms written
// out separately there, and here).
template <typename R>
__device__ __forceinline__ void c2op(Cx<R>& c, int eqop, int kind, Cx<R> a, Cx<R> b) {
  if (kind == 4) {
    switch (eqop) {
      case EQ: c = a; return;
      case EQM: c.re = -a.re; c.im = -a.im; return;
      case PEQ: c.re = radd(c.re, a.re); c.im = radd(c.im, a.im); return;
      default: c.re = rsub(c.re, a.re); c.im = rsub(c.im, a.im); return;
    }
  }
  if (eqop == EQM) {
    switch (kind) {
      case 0: c.re = rsub(-a.re, b.re); c.im = rsub(-a.im, b.im); return;
      case 1: c.re = radd(-a.re, b.re); c.im = radd(-a.im, b.im); return;
      case 2: c.re = radd(-a.re, b.im); c.im = rsub(-a.im, b.re); return;
      default: c.re = rsub(-a.re, b.im); c.im = radd(-a.im, b.re); return;
    }
  }
  R re, im;
  switch (kind) {
    case 0: re = radd(a.re, b.re); im = radd(a.im, b.im); break;
    case 1: re = rsub(a.re, b.re); im = rsub(a.im, b.im); break;
    case 2: re = rsub(a.re, b.im); im = radd(a.im, b.re); break;
    default: re = radd(a.re, b.im); im = rsub(a.im, b.re); break;
  }
  if (eqop == EQ) {
    c.re = re;
    c.im = im;
  } else if (eqop == PEQ) {
    c.re = radd(c.re, re);
    c.im = radd(c.im, im);
  } else {
    c.re = rsub(c.re, re);
    c.im = rsub(c.im, im);
  }
}

// one-operand op of the reconstruction through the carith1 table
// (lib/perl/headers.pl:136-169) onto qla_complex.h:147-172.
template <typename R>
__device__ __forceinline__ void c1op(Cx<R>& c, int eqop, int op, Cx<R> a) {
  if (op == 0) {
    if (eqop == EQ || eqop == EQM) {
      c.re = R(0);
      c.im = R(0);
    }
    return;
  }
  const bool neg = (op == 2 || op == 4);
  const bool ic = (op == 3 || op == 4);
  int e = eqop;
  if (neg) e = (eqop == EQ) ? EQM : (eqop == EQM) ? EQ : (eqop == PEQ) ? MEQ : PEQ;
  if (!ic) {
    switch (e) {
      case EQ: c = a; break;
      case EQM: c.re = -a.re; c.im = -a.im; break;
      case PEQ: c.re = radd(c.re, a.re); c.im = radd(c.im, a.im); break;
      default: c.re = rsub(c.re, a.re); c.im = rsub(c.im, a.im); break;
    }
  } else {
    switch (e) {
      case EQ: c.re = -a.im; c.im = a.re; break;
      case EQM: c.re = a.im; c.im = -a.re; break;
      case PEQ: c.re = rsub(c.re, a.im); c.im = radd(c.im, a.re); break;
      default: c.re = radd(c.re, a.im); c.im = rsub(c.im, a.re); break;
    }
  }
}

// Host-visible copies of the tables for compile-time dispatch.
struct SpinTables {
  static constexpr signed char spproj[2][5][2][3] = {
      {{{2, 0, 3}, {2, 1, 2}}, {{1, 0, 3}, {0, 1, 2}}, {{2, 0, 2}, {3, 1, 3}}, {{0, 0, 2}, {0, 1, 3}},
       {{4, 0, 0}, {4, 1, 1}}},
      {{{3, 0, 3}, {3, 1, 2}}, {{0, 0, 3}, {1, 1, 2}}, {{3, 0, 2}, {2, 1, 3}}, {{1, 0, 2}, {1, 1, 3}},
       {{4, 2, 2}, {4, 3, 3}}}};
  static constexpr signed char sprecon[2][5][4][2] = {
      {{{1, 0}, {1, 1}, {4, 1}, {4, 0}},
       {{1, 0}, {1, 1}, {1, 1}, {2, 0}},
       {{1, 0}, {1, 1}, {4, 0}, {3, 1}},
       {{1, 0}, {1, 1}, {1, 0}, {1, 1}},
       {{1, 0}, {1, 1}, {0, 0}, {0, 1}}},
      {{{1, 0}, {1, 1}, {3, 1}, {3, 0}},
       {{1, 0}, {1, 1}, {2, 1}, {1, 0}},
       {{1, 0}, {1, 1}, {3, 0}, {4, 1}},
       {{1, 0}, {1, 1}, {2, 0}, {2, 1}},
       {{0, 0}, {0, 1}, {1, 0}, {1, 1}}}};
};

// Dispatch a runtime (mu, sign) pair onto a compile-time body F::run<MU, SG>
// so that every spin index is a constant (no dynamic register indexing).
template <class F, class... A>
__device__ __forceinline__ void mu_sign_dispatch(int mu, int sign, A&&... args) {
  const int sg = (sign == 1) ? 0 : 1;
  switch (mu * 2 + sg) {
    case 0: F::template run<0, 0>(args...); break;
    case 1: F::template run<0, 1>(args...); break;
    case 2: F::template run<1, 0>(args...); break;
    case 3: F::template run<1, 1>(args...); break;
    case 4: F::template run<2, 0>(args...); break;
    case 5: F::template run<2, 1>(args...); break;
    case 6: F::template run<3, 0>(args...); break;
    case 7: F::template run<3, 1>(args...); break;
    case 8: F::template run<4, 0>(args...); break;
    default: F::template run<4, 1>(args...); break;
  }
}

// H (eqop) spproj(D, mu, sign): build_qla.pl:1087-1110, make_code_unary.pl:183-241.
// (mu outside 0..4 is a no-op in the reference; the host never launches it.)
template <typename R_, int NC>
struct SpprojOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = NC * 4, N1 = 0, N2 = 0, NOUT = NC * 2, NACC = 0;
  struct Body {
    template <int MU, int SG, int LA, int LY>
    __device__ __forceinline__ static void run(int eqop, const Cx<R> (&a)[LA], Cx<R> (&y)[LY]) {
      static_assert(LA >= N0 && LY >= NOUT, "record array too short");
      constexpr int k0 = SpinTables::spproj[SG][MU][0][0], a0 = SpinTables::spproj[SG][MU][0][1],
                    b0 = SpinTables::spproj[SG][MU][0][2];
      constexpr int k1 = SpinTables::spproj[SG][MU][1][0], a1 = SpinTables::spproj[SG][MU][1][1],
                    b1 = SpinTables::spproj[SG][MU][1][2];
#pragma unroll
      for (int ic = 0; ic < NC; ic++) {
        c2op(y[ic * 2 + 0], eqop, k0, a[ic * 4 + a0], a[ic * 4 + b0]);
        c2op(y[ic * 2 + 1], eqop, k1, a[ic * 4 + a1], a[ic * 4 + b1]);
      }
    }
  };
  __device__ __forceinline__ static void apply(const SiteParams& p, const Cx<R> (&a)[N0], const Cx<R> (&)[1],
                                               const Cx<R> (&)[1], Cx<R> (&y)[NOUT]) {
    mu_sign_dispatch<Body>(p.mu, p.sign, p.eqop, a, y);
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[N0], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

// D (eqop) sprecon(H, mu, sign): build_qla.pl:1112-1135
template <typename R_, int NC>
struct SpreconOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = NC * 2, N1 = 0, N2 = 0, NOUT = NC * 4, NACC = 0;
  struct Body {
    template <int MU, int SG, int LH, int LY>
    __device__ __forceinline__ static void run(int eqop, const Cx<R> (&h)[LH], Cx<R> (&y)[LY]) {
      static_assert(LH >= N0 && LY >= NOUT, "record array too short");
      constexpr int o0 = SpinTables::sprecon[SG][MU][0][0], s0 = SpinTables::sprecon[SG][MU][0][1];
      constexpr int o1 = SpinTables::sprecon[SG][MU][1][0], s1 = SpinTables::sprecon[SG][MU][1][1];
      constexpr int o2 = SpinTables::sprecon[SG][MU][2][0], s2 = SpinTables::sprecon[SG][MU][2][1];
      constexpr int o3 = SpinTables::sprecon[SG][MU][3][0], s3 = SpinTables::sprecon[SG][MU][3][1];
#pragma unroll
      for (int ic = 0; ic < NC; ic++) {
        c1op(y[ic * 4 + 0], eqop, o0, h[ic * 2 + s0]);
        c1op(y[ic * 4 + 1], eqop, o1, h[ic * 2 + s1]);
        c1op(y[ic * 4 + 2], eqop, o2, h[ic * 2 + s2]);
        c1op(y[ic * 4 + 3], eqop, o3, h[ic * 2 + s3]);
      }
    }
  };
  __device__ __forceinline__ static void apply(const SiteParams& p, const Cx<R> (&h)[N0], const Cx<R> (&)[1],
                                               const Cx<R> (&)[1], Cx<R> (&y)[NOUT]) {
    mu_sign_dispatch<Body>(p.mu, p.sign, p.eqop, h, y);
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[N0], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

// ---------------------------------------------------------------------------
// Fused spin-projection / colour-multiply / reconstruction (the Wilson hop
// terms), build_qla.pl:1137-1250, make_code_binary.pl:189-336: the
// intermediates are formed with `eq` exactly as the reference's temporaries
// t1, t2, and only the last step applies the eqop.
//   DEST = 2 (H):  r (eqop) A * spproj(b)
//   DEST = 4 (D):  r (eqop) sprecon(A * spproj(b))
template <typename R_, int NC, bool ADJA, int DEST>
struct SpprojMultOp {
  using R = R_;
  static constexpr int NIN = 2, N0 = NC * NC, N1 = NC * 4, N2 = 0, NOUT = NC * DEST, NACC = 0;
  __device__ __forceinline__ static void apply(const SiteParams& p, const Cx<R> (&a)[N0], const Cx<R> (&b)[N1],
                                               const Cx<R> (&)[1], Cx<R> (&y)[NOUT]) {
    Cx<R> t1[NC * 2];
    mu_sign_dispatch<typename SpprojOp<R, NC>::Body>(p.mu, p.sign, (int)EQ, b, t1);
    if constexpr (DEST == 2) {
      lmult_site<R, NC, 2, ADJA, false>(p.eqop, p.out_read != 0, a, t1, y);
    } else {
      Cx<R> t2[NC * 2];
      lmult_site<R, NC, 2, ADJA, false>(EQ, false, a, t1, t2);
      mu_sign_dispatch<typename SpreconOp<R, NC>::Body>(p.mu, p.sign, p.eqop, t2, y);
    }
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[N0], const Cx<R> (&)[N1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

// r (eqop) sprecon(A * b), b a HalfFermion (build_qla.pl:1200-1250)
template <typename R_, int NC, bool ADJA>
struct SpreconMultOp {
  using R = R_;
  static constexpr int NIN = 2, N0 = NC * NC, N1 = NC * 2, N2 = 0, NOUT = NC * 4, NACC = 0;
  __device__ __forceinline__ static void apply(const SiteParams& p, const Cx<R> (&a)[N0], const Cx<R> (&b)[N1],
                                               const Cx<R> (&)[1], Cx<R> (&y)[NOUT]) {
    Cx<R> t[NC * 2];
    lmult_site<R, NC, 2, ADJA, false>(EQ, false, a, b, t);
    mu_sign_dispatch<typename SpreconOp<R, NC>::Body>(p.mu, p.sign, p.eqop, t, y);
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[N0], const Cx<R> (&)[N1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

// D (eqop) spproj(D): projection onto the D record (build_qla.pl:1137-1160)
template <typename R_, int NC>
struct SpprojDOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = NC * 4, N1 = 0, N2 = 0, NOUT = NC * 4, NACC = 0;
  __device__ __forceinline__ static void apply(const SiteParams& p, const Cx<R> (&b)[N0], const Cx<R> (&)[1],
                                               const Cx<R> (&)[1], Cx<R> (&y)[NOUT]) {
    Cx<R> t[NC * 2];
    mu_sign_dispatch<typename SpprojOp<R, NC>::Body>(p.mu, p.sign, (int)EQ, b, t);
    mu_sign_dispatch<typename SpreconOp<R, NC>::Body>(p.mu, p.sign, p.eqop, t, y);
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[N0], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

// ---------------------------------------------------------------------------
// r (eqop) a * b with a real scalar: build_qla.pl:1256-1292,
// qla_complex.h:258-265 (scalar read once as `at = *a`).
template <typename R>
__device__ __forceinline__ R scalar_arg(const SiteParams& p) {
  if (p.sptr) return __ldg(static_cast<const R*>(p.sptr));
  return static_cast<R>(p.sval);
}

template <typename R_, int NCPLX>
struct RTimesOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = NCPLX, N1 = 0, N2 = 0, NOUT = NCPLX, NACC = 0;
  __device__ __forceinline__ static void apply(const SiteParams& p, const Cx<R> (&b)[N0], const Cx<R> (&)[1],
                                               const Cx<R> (&)[1], Cx<R> (&y)[NOUT]) {
    const R at = scalar_arg<R>(p);
#pragma unroll
    for (int e = 0; e < NCPLX; e++) {
      const R pr = rmul(at, b[e].re), pi = rmul(at, b[e].im);
      switch (p.eqop) {
        case EQ: y[e].re = pr; y[e].im = pi; break;
        case EQM: y[e].re = -pr; y[e].im = -pi; break;
        case PEQ: y[e].re = radd(y[e].re, pr); y[e].im = radd(y[e].im, pi); break;
        default: y[e].re = rsub(y[e].re, pr); y[e].im = rsub(y[e].im, pi); break;
      }
    }
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[N0], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

// r (eqop) b : copies and gathers (build_qla.pl:370-400, V_veq_pV / V_eq_xV)
template <typename R_, int NCPLX>
struct CopyOp {
  using R = R_;
  static constexpr int NIN = 1, N0 = NCPLX, N1 = 0, N2 = 0, NOUT = NCPLX, NACC = 0;
  __device__ __forceinline__ static void apply(const SiteParams& p, const Cx<R> (&b)[N0], const Cx<R> (&)[1],
                                               const Cx<R> (&)[1], Cx<R> (&y)[NOUT]) {
#pragma unroll
    for (int e = 0; e < NCPLX; e++) {
      switch (p.eqop) {
        case EQ: y[e] = b[e]; break;
        case EQM: y[e].re = -b[e].re; y[e].im = -b[e].im; break;
        case PEQ: y[e].re = radd(y[e].re, b[e].re); y[e].im = radd(y[e].im, b[e].im); break;
        default: y[e].re = rsub(y[e].re, b[e].re); y[e].im = rsub(y[e].im, b[e].im); break;
      }
    }
  }
  __device__ static void accum(const SiteParams&, const Cx<R> (&)[N0], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               double*) {}
  __device__ static void finish(const SiteParams&, const double*) {}
};

// ---------------------------------------------------------------------------
// Global reductions (build_qla.pl:2089-2155 norm2, 2196-2360 dot).  The
// reference sums sequentially in double; here every product of two inputs is
// formed in double (exact for float inputs), summed per site in double and
// accumulated across sites in double-double, then rounded once to the
// destination type OUT (float for F3, double for DF3/D3).
template <typename OUT>
__device__ __forceinline__ void write_real(const SiteParams& p, double v) {
  *static_cast<OUT*>(p.result) = static_cast<OUT>(v);
}
template <typename OUT>
__device__ __forceinline__ void write_cplx(const SiteParams& p, double re, double im) {
  OUT* r = static_cast<OUT*>(p.result);
  r[0] = static_cast<OUT>(re);
  r[1] = static_cast<OUT>(im);
}

template <typename R_, int NCPLX, typename OUT>
struct Norm2Op {
  using R = R_;
  static constexpr int NIN = 1, N0 = NCPLX, N1 = 0, N2 = 0, NOUT = 0, NACC = 1;
  __device__ static void apply(const SiteParams&, const Cx<R> (&)[N0], const Cx<R> (&)[1], const Cx<R> (&)[1],
                               Cx<R> (&)[1]) {}
  __device__ __forceinline__ static void accum(const SiteParams&, const Cx<R> (&a)[N0], const Cx<R> (&)[1],
                                               const Cx<R> (&)[1], double* acc) {
    double s = 0.0;
#pragma unroll
    for (int e = 0; e < NCPLX; e++) {
      const double re = a[e].re, im = a[e].im;
      s = __dadd_rn(s, __dadd_rn(__dmul_rn(re, re), __dmul_rn(im, im)));
    }
    acc[0] = s;
  }
  __device__ static void finish(const SiteParams& p, const double* tot) { write_real<OUT>(p, tot[0]); }
};

template <typename R_, int NCPLX, typename OUT>
struct DotOp {
  using R = R_;
  static constexpr int NIN = 2, N0 = NCPLX, N1 = NCPLX, N2 = 0, NOUT = 0, NACC = 2;
  __device__ static void apply(const SiteParams&, const Cx<R> (&)[N0], const Cx<R> (&)[N1], const Cx<R> (&)[1],
                               Cx<R> (&)[1]) {}
  __device__ __forceinline__ static void accum(const SiteParams&, const Cx<R> (&a)[N0], const Cx<R> (&b)[N1],
                                               const Cx<R> (&)[1], double* acc) {
    double sr = 0.0, si = 0.0;
#pragma unroll
    for (int e = 0; e < NCPLX; e++) {
      const double ar = a[e].re, ai = a[e].im, br = b[e].re, bi = b[e].im;
      sr = __dadd_rn(sr, __dadd_rn(__dmul_rn(ar, br), __dmul_rn(ai, bi)));
      si = __dadd_rn(si, __dsub_rn(__dmul_rn(ar, bi), __dmul_rn(ai, br)));
    }
    acc[0] = sr;
    acc[1] = si;
  }
  __device__ static void finish(const SiteParams& p, const double* tot) { write_cplx<OUT>(p, tot[0], tot[1]); }
};

// real part of the inner product (r_veq_re_X_dot_X, build_qla.pl:1809 / 2250)
template <typename R_, int NCPLX, typename OUT>
struct ReDotOp {
  using R = R_;
  static constexpr int NIN = 2, N0 = NCPLX, N1 = NCPLX, N2 = 0, NOUT = 0, NACC = 1;
  __device__ static void apply(const SiteParams&, const Cx<R> (&)[N0], const Cx<R> (&)[N1], const Cx<R> (&)[1],
                               Cx<R> (&)[1]) {}
  __device__ __forceinline__ static void accum(const SiteParams&, const Cx<R> (&a)[N0], const Cx<R> (&b)[N1],
                                               const Cx<R> (&)[1], double* acc) {
    double sr = 0.0;
#pragma unroll
    for (int e = 0; e < NCPLX; e++) {
      const double ar = a[e].re, ai = a[e].im, br = b[e].re, bi = b[e].im;
      sr = __dadd_rn(sr, __dadd_rn(__dmul_rn(ar, br), __dmul_rn(ai, bi)));
    }
    acc[0] = sr;
  }
  __device__ static void finish(const SiteParams& p, const double* tot) { write_real<OUT>(p, tot[0]); }
};

}  // namespace qlab
