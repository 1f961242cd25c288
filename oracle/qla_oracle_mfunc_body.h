/*
 * Test infrastructure (the oracle): restatement of QLA's matrix-function code
 * templates (the C files under lib/perl/code-templates), precision-generic.  Included twice
 * by qla_oracle_mfunc.c with R = float / double and SFX = f / d, mirroring the
 * reference's F and D builds of the same templates.  nc is a run-time colour
 * count (<= ORA_NCMAX), as in the reference's N-colour build; for nc == 2 and 3 the
 * closed forms of the templates are used where the templates have them.
 *
 * Every helper restates the generated level-1 function the template calls
 * (QLA_<P><C>_M_eq_M_times_M, M_peq_r_times_M, ...), in its operation order.
 */

#define CAT2_(a, b) a##_##b
#define CAT2(a, b) CAT2_(a, b)
#define FN(name) CAT2(name, SFX)

typedef struct { R re, im; } FN(mc);

#define EL(m, i, j) ((m)[(i) * nc + (j)])

/* M_eq_c with a real constant: diagonal d, off-diagonal 0 (QLA_F3_M_eq_c) */
static void FN(m_eq_d)(FN(mc) *r, int nc, R d)
{
  for (int i = 0; i < nc; i++) {
    for (int j = 0; j < nc; j++) { EL(r, i, j).re = 0.; EL(r, i, j).im = 0.; }
    EL(r, i, i).re = d; EL(r, i, i).im = 0.;
  }
}

/* r += s * a  (QLA_F3_M_peq_r_times_M, qla_complex.h:262) */
static void FN(m_peq_r_times_m)(FN(mc) *r, int nc, R s, const FN(mc) *a)
{
  for (int k = 0; k < nc * nc; k++) { r[k].re += s * a[k].re; r[k].im += s * a[k].im; }
}

/* r = s * a  (QLA_F3_M_eq_r_times_M) */
static void FN(m_eq_r_times_m)(FN(mc) *r, int nc, R s, const FN(mc) *a)
{
  for (int k = 0; k < nc * nc; k++) { r[k].re = s * a[k].re; r[k].im = s * a[k].im; }
}

/* r = a * b  (QLA_F3_M_eq_M_times_M: x = 0; x += a_ik b_kj in k order) */
static void FN(m_eq_m_times_m)(FN(mc) *r, int nc, const FN(mc) *a, const FN(mc) *b)
{
  for (int i = 0; i < nc; i++)
    for (int j = 0; j < nc; j++) {
      R xr = 0., xi = 0.;
      for (int k = 0; k < nc; k++) {
        FN(mc) u = EL(a, i, k), v = EL(b, k, j);
        xr += (u.re * v.re - u.im * v.im);
        xi += (u.re * v.im + u.im * v.re);
      }
      EL(r, i, j).re = xr; EL(r, i, j).im = xi;
    }
}

/* sum |a_ij|^2 with each term in R, promoted and summed in double
 * (maxev2 of M_eq_sqrt_M.c:60-70; maxev of M_eq_exp_M.c:76-87 is its sqrt) */
static double FN(fnorm2)(const FN(mc) *a, int nc)
{
  double s = 0.;
  for (int k = 0; k < nc * nc; k++) s += a[k].re * a[k].re + a[k].im * a[k].im;
  return s;
}

/* x = a^-1 b by Gauss-Jordan elimination with partial pivoting
 * (M_eq_M_inverse_M.c:108-135; also the generic path of M_eq_inverse_M.c:120-162
 * with b = 1).  Rows are swapped physically; the arithmetic is the same as
 * the template's row-permutation form. */
static void FN(m_eq_m_inverse_m)(FN(mc) *x, int nc, const FN(mc) *a, const FN(mc) *b, int nb)
{
  FN(mc) c[ORA_NCMAX * ORA_NCMAX], d[ORA_NCMAX * ORA_NCMAX];
  int row[ORA_NCMAX];
  for (int i = 0; i < nc; i++) {
    for (int j = 0; j < nc; j++) EL(c, i, j) = EL(a, i, j);
    for (int j = 0; j < nb; j++) d[i * nb + j] = b[i * nb + j];
    row[i] = i;
  }
#define CC(i, j) EL(c, row[i], j)
#define DD(i, j) d[row[i] * nb + (j)]
  for (int k = 0; k < nc; k++) {
    R rmax = CC(k, k).re * CC(k, k).re + CC(k, k).im * CC(k, k).im;
    int imax = k;
    for (int i = k + 1; i < nc; i++) {
      R rr = CC(i, k).re * CC(i, k).re + CC(i, k).im * CC(i, k).im;
      if (rr > rmax) { rmax = rr; imax = i; }
    }
    { int rk = row[k]; row[k] = row[imax]; row[imax] = rk; }
    rmax = 1 / rmax;
    FN(mc) s;                                   /* QLA_c_eq_r_times_ca, qla_complex.h:272 */
    s.re = rmax * CC(k, k).re;
    s.im = -(rmax * CC(k, k).im);
    CC(k, k) = s;
    for (int i = 0; i < nc; i++) {
      if (i == k) continue;
      FN(mc) t;
      t.re = s.re * CC(i, k).re - s.im * CC(i, k).im;
      t.im = s.re * CC(i, k).im + s.im * CC(i, k).re;
      for (int j = k + 1; j < nc; j++) {
        CC(i, j).re -= (t.re * CC(k, j).re - t.im * CC(k, j).im);
        CC(i, j).im -= (t.re * CC(k, j).im + t.im * CC(k, j).re);
      }
      for (int j = 0; j < nb; j++) {
        DD(i, j).re -= (t.re * DD(k, j).re - t.im * DD(k, j).im);
        DD(i, j).im -= (t.re * DD(k, j).im + t.im * DD(k, j).re);
      }
    }
  }
  for (int i = 0; i < nc; i++)
    for (int j = 0; j < nb; j++) {
      FN(mc) u = CC(i, i), v = DD(i, j);
      x[i * nb + j].re = u.re * v.re - u.im * v.im;
      x[i * nb + j].im = u.re * v.im + u.im * v.re;
    }
#undef CC
#undef DD
}

/* ------------------------------------------------------------------ det */
/* C_eq_det_M.c:70-84 (nc = 3 cofactor expansion), :86-143 (LU, generic) */
static void FN(det1)(FN(mc) *out, const FN(mc) *a, int nc)
{
#define CMUL(r, p, q) { (r).re = (p).re * (q).re - (p).im * (q).im; (r).im = (p).re * (q).im + (p).im * (q).re; }
#define CMMS(r, p, q) { (r).re -= ((p).re * (q).re - (p).im * (q).im); (r).im -= ((p).re * (q).im + (p).im * (q).re); }
#define CPMS(r, p, q) { (r).re += ((p).re * (q).re - (p).im * (q).im); (r).im += ((p).re * (q).im + (p).im * (q).re); }
  if (nc == 3) {
    FN(mc) det, det0, det1, det2;
    CMUL(det2, EL(a, 0, 0), EL(a, 1, 1)); CMMS(det2, EL(a, 0, 1), EL(a, 1, 0));
    CMUL(det1, EL(a, 0, 2), EL(a, 1, 0)); CMMS(det1, EL(a, 0, 0), EL(a, 1, 2));
    CMUL(det0, EL(a, 0, 1), EL(a, 1, 2)); CMMS(det0, EL(a, 0, 2), EL(a, 1, 1));
    CMUL(det, det2, EL(a, 2, 2));
    CPMS(det, det1, EL(a, 2, 1));
    CPMS(det, det0, EL(a, 2, 0));
    *out = det;
    return;
  }
  FN(mc) c[ORA_NCMAX * ORA_NCMAX];
  int row[ORA_NCMAX], nswaps = 0;
  FN(mc) x; x.re = 1; x.im = 0.;
  for (int i = 0; i < nc; i++) { for (int j = 0; j < nc; j++) EL(c, i, j) = EL(a, i, j); row[i] = i; }
#define CC(i, j) EL(c, row[i], j)
  for (int j = 0; j < nc; j++) {
    if (j > 0) {
      for (int i = j; i < nc; i++) {
        FN(mc) t2 = CC(i, j);
        for (int k = 0; k < j; k++) CMMS(t2, CC(i, k), CC(k, j));
        CC(i, j) = t2;
      }
    }
    R rmax = CC(j, j).re * CC(j, j).re + CC(j, j).im * CC(j, j).im;
    int kmax = j;
    for (int k = j + 1; k < nc; k++) {
      R rr = CC(k, j).re * CC(k, j).re + CC(k, j).im * CC(k, j).im;
      if (rr > rmax) { rmax = rr; kmax = k; }
    }
    if (rmax == 0) { out->re = 0; out->im = 0.; return; }
    if (kmax != j) { int rj = row[j]; row[j] = row[kmax]; row[kmax] = rj; nswaps++; }
    { FN(mc) z = x; CMUL(x, z, CC(j, j)); }
    R ri = 1 / rmax;
    FN(mc) cjji; cjji.re = ri * CC(j, j).re; cjji.im = -(ri * CC(j, j).im);
    for (int i = j + 1; i < nc; i++) {
      FN(mc) t2 = CC(j, i);
      for (int k = 0; k < j; k++) CMMS(t2, CC(j, k), CC(k, i));
      CMUL(CC(j, i), t2, cjji);
    }
  }
  if (nswaps & 1) { x.re = -x.re; x.im = -x.im; }
  *out = x;
#undef CC
}

/* -------------------------------------------------------------- inverse */
/* M_eq_inverse_M.c:79-119 (nc = 3 cofactors), :120-162 (Gauss-Jordan) */
static void FN(inverse1)(FN(mc) *x, const FN(mc) *a, int nc)
{
  if (nc == 3) {
    FN(mc) det0, det1, det2, det, idet;
    CMUL(det2, EL(a, 0, 0), EL(a, 1, 1)); CMMS(det2, EL(a, 0, 1), EL(a, 1, 0));
    CMUL(det1, EL(a, 0, 2), EL(a, 1, 0)); CMMS(det1, EL(a, 0, 0), EL(a, 1, 2));
    CMUL(det0, EL(a, 0, 1), EL(a, 1, 2)); CMMS(det0, EL(a, 0, 2), EL(a, 1, 1));
    CMUL(det, det2, EL(a, 2, 2));
    CPMS(det, det1, EL(a, 2, 1));
    CPMS(det, det0, EL(a, 2, 0));
    {                                   /* QLA_c_eq_r_div_c(idet, 1, det), qla_complex.h */
      R t = (R)1 / (det.re * det.re + det.im * det.im);
      idet.re = t * det.re;
      idet.im = -t * det.im;
    }
#define SET(i0, j0, i1, j1, i2, j2) \
    CMUL(det, EL(a, i1, j1), EL(a, i2, j2)); CMMS(det, EL(a, i1, j2), EL(a, i2, j1)); CMUL(EL(x, i0, j0), det, idet);
    SET(0, 0, 1, 1, 2, 2);
    SET(0, 1, 2, 1, 0, 2);
    CMUL(EL(x, 0, 2), det0, idet);
    SET(1, 0, 1, 2, 2, 0);
    SET(1, 1, 2, 2, 0, 0);
    CMUL(EL(x, 1, 2), det1, idet);
    SET(2, 0, 1, 0, 2, 1);
    SET(2, 1, 2, 0, 0, 1);
    CMUL(EL(x, 2, 2), det2, idet);
#undef SET
    return;
  }
  FN(mc) one[ORA_NCMAX * ORA_NCMAX] = {{0}};
  FN(m_eq_d)(one, nc, 1);
  FN(m_eq_m_inverse_m)(x, nc, a, one, nc);
}

/* ------------------------------------------------------------------ exp */
/* M_eq_exp_M.c:302-367: generic path (OPT_NC3 is disabled, :12), scaling by
 * s = ceil(2 |a|_F) <= 1024, rational approximation with P, Q (:61-72),
 * binary powering. */
static const double FN(padeP)[] = {9.99999999999999999910E-1, 3.02994407707441961300E-2,
                                   1.26177193074810590878E-4};
static const double FN(padeQ)[] = {2.00000000000000000009E0, 2.27265548208155028766E-1,
                                   2.52448340349684104192E-3, 3.00198505138664455042E-6};

static void FN(exp1)(FN(mc) *r, const FN(mc) *a, int nc)
{
  double ds = sqrt(FN(fnorm2)(a, nc));
  if (ds == 0) { FN(m_eq_d)(r, nc, 1); return; }
  unsigned int s = (unsigned int)ceil(2 * ds);
  if (s > 1024) s = 1024;
  ds = (double)s;
  FN(mc) bs[ORA_NCMAX * ORA_NCMAX], bs2[ORA_NCMAX * ORA_NCMAX], bs4[ORA_NCMAX * ORA_NCMAX],
      bs6[ORA_NCMAX * ORA_NCMAX], pb[ORA_NCMAX * ORA_NCMAX], qb[ORA_NCMAX * ORA_NCMAX];
  R dsi = 1.0 / ds;
  FN(m_eq_r_times_m)(bs, nc, dsi, a);
  FN(m_eq_d)(pb, nc, (R)FN(padeP)[0]);
  FN(m_eq_d)(qb, nc, (R)FN(padeQ)[0]);
  FN(m_eq_m_times_m)(bs2, nc, bs, bs);
  FN(m_peq_r_times_m)(pb, nc, (R)FN(padeP)[1], bs2);
  FN(m_peq_r_times_m)(qb, nc, (R)FN(padeQ)[1], bs2);
  FN(m_eq_m_times_m)(bs4, nc, bs2, bs2);
  FN(m_peq_r_times_m)(pb, nc, (R)FN(padeP)[2], bs4);
  FN(m_peq_r_times_m)(qb, nc, (R)FN(padeQ)[2], bs4);
  FN(m_eq_m_times_m)(bs6, nc, bs4, bs2);
  FN(m_peq_r_times_m)(qb, nc, (R)FN(padeQ)[3], bs6);
  FN(m_eq_m_times_m)(bs6, nc, bs, pb);
  for (int k = 0; k < nc * nc; k++) {            /* M_eq_M_minus_M */
    pb[k].re = qb[k].re - bs6[k].re;
    pb[k].im = qb[k].im - bs6[k].im;
  }
  FN(m_eq_m_inverse_m)(qb, nc, pb, bs6, nc);
  FN(m_eq_d)(pb, nc, 1);
  FN(m_peq_r_times_m)(pb, nc, (R)2, qb);
  if (s == 1) { memcpy(r, pb, sizeof(FN(mc)) * nc * nc); return; }
  FN(mc) *va0 = bs, *va1 = bs2, *vb0 = pb, *vb1 = bs6, *tmp;
  FN(m_eq_d)(va0, nc, 1);
  for (; s > 0; s >>= 1) {
    if (s & 1) { FN(m_eq_m_times_m)(va1, nc, va0, vb0); tmp = va1; va1 = va0; va0 = tmp; }
    if (s > 0) { FN(m_eq_m_times_m)(vb1, nc, vb0, vb0); tmp = vb1; vb1 = vb0; vb0 = tmp; }
  }
  memcpy(r, va0, sizeof(FN(mc)) * nc * nc);
}

/* ----------------------------------------------------------------- sqrt */
/* M_eq_sqrt_M.c:139-180: Newton iteration e <- -1/2 e x^-1 e, x += e, until
 * |e|_F^2 <= EPS (FLT_EPSILON / DBL_EPSILON) or 20 iterations. */
/* Newton loop shared by sqrt and invsqrt (M_eq_sqrt_M.c:158-171,
 * M_eq_invsqrt_M.c:160-173): e <- -1/2 e x^-1 e, x += e. */
static void FN(newton_sqrt)(FN(mc) *x, FN(mc) *e, int nc, double eps)
{
  FN(mc) t1[ORA_NCMAX * ORA_NCMAX], t2[ORA_NCMAX * ORA_NCMAX];
  double enorm;
  int nit = 0;
  do {
    nit++;
    FN(m_eq_m_inverse_m)(t1, nc, x, e, nc);
    FN(m_eq_m_times_m)(t2, nc, e, t1);
    FN(m_eq_r_times_m)(e, nc, (R)(-0.5), t2);
    for (int k = 0; k < nc * nc; k++) { x[k].re += e[k].re; x[k].im += e[k].im; }
    enorm = FN(fnorm2)(e, nc);
  } while (nit < 20 && enorm > eps);
}

static void FN(sqrt1)(FN(mc) *r, const FN(mc) *a, int nc, double eps)
{
  double ds = FN(fnorm2)(a, nc);
  if (ds == 0) { FN(m_eq_d)(r, nc, 0); return; }
  ds = sqrt(ds);
  FN(mc) x[ORA_NCMAX * ORA_NCMAX], e[ORA_NCMAX * ORA_NCMAX];
  FN(m_eq_r_times_m)(x, nc, (R)(1 / ds), a);
  FN(m_eq_d)(e, nc, (R)0.5);
  FN(m_peq_r_times_m)(e, nc, (R)(-0.5), x);
  for (int k = 0; k < nc * nc; k++) { x[k].re += e[k].re; x[k].im += e[k].im; }
  FN(newton_sqrt)(x, e, nc, eps);
  FN(m_eq_r_times_m)(r, nc, (R)sqrt(ds), x);
}

/* -------------------------------------------------------------- invsqrt */
/* M_eq_invsqrt_M.c:88-127: the same Newton iteration started from
 * x = 1, e = 0.5 ds a^-1 - 0.5; a zero matrix gives 1/0 on the diagonal. */
static void FN(invsqrt1)(FN(mc) *r, const FN(mc) *a, int nc, double eps)
{
  double ds = FN(fnorm2)(a, nc);
  if (ds == 0) { FN(m_eq_d)(r, nc, (R)INFINITY); return; }
  ds = sqrt(ds);
  FN(mc) x[ORA_NCMAX * ORA_NCMAX], e[ORA_NCMAX * ORA_NCMAX], xi[ORA_NCMAX * ORA_NCMAX];
  FN(m_eq_d)(x, nc, 1);
  FN(inverse1)(xi, a, nc);
  FN(m_eq_d)(e, nc, (R)(-0.5));
  FN(m_peq_r_times_m)(e, nc, (R)(0.5 * ds), xi);
  for (int k = 0; k < nc * nc; k++) { x[k].re += e[k].re; x[k].im += e[k].im; }
  FN(newton_sqrt)(x, e, nc, eps);
  FN(m_eq_r_times_m)(r, nc, (R)(1 / sqrt(ds)), x);
}

/* ------------------------------------------------------------------ log */
/* M_eq_log_M.c:127-199 (every nc > 2): scale by 1/|a|_F, four square roots,
 * log(1 + x) = x - x^2/2 + x^3 P(x)/Q(x) with the coefficients of :52-68,
 * times 2^4, plus log|a|_F on the diagonal. */
static const double FN(logP)[] = {7.70838733755885391666E0, 1.79368678507819816313E1,
                                  1.44989225341610930846E1, 4.70579119878881725854E0,
                                  4.97494994976747001425E-1, 1.01875663804580931796E-4};
static const double FN(logQ)[] = {2.31251620126765340583E1, 7.11544750618563894466E1,
                                  8.29875266912776603211E1, 4.52279145837532221105E1,
                                  1.12873587189167450590E1};

static void FN(log1)(FN(mc) *r, const FN(mc) *a, int nc, double eps)
{
  double ds = sqrt(FN(fnorm2)(a, nc));
  if (ds == 0) { FN(m_eq_d)(r, nc, (R)log(0.)); return; }
  FN(mc) as[ORA_NCMAX * ORA_NCMAX], as2[ORA_NCMAX * ORA_NCMAX], as3[ORA_NCMAX * ORA_NCMAX],
      as4[ORA_NCMAX * ORA_NCMAX], as5[ORA_NCMAX * ORA_NCMAX], pa[ORA_NCMAX * ORA_NCMAX],
      qa[ORA_NCMAX * ORA_NCMAX];
  FN(m_eq_r_times_m)(as, nc, (R)(1 / ds), a);
  for (int i = 0; i < 4; i++) {
    memcpy(as2, as, sizeof(FN(mc)) * nc * nc);
    FN(sqrt1)(as, as2, nc, eps);
  }
  for (int i = 0; i < nc; i++) EL(as, i, i).re -= 1;
  FN(m_eq_d)(pa, nc, (R)FN(logP)[0]);
  FN(m_eq_d)(qa, nc, (R)FN(logQ)[0]);
  FN(m_peq_r_times_m)(pa, nc, (R)FN(logP)[1], as);
  FN(m_peq_r_times_m)(qa, nc, (R)FN(logQ)[1], as);
  FN(m_eq_m_times_m)(as2, nc, as, as);
  FN(m_peq_r_times_m)(pa, nc, (R)FN(logP)[2], as2);
  FN(m_peq_r_times_m)(qa, nc, (R)FN(logQ)[2], as2);
  FN(m_eq_m_times_m)(as3, nc, as, as2);
  FN(m_peq_r_times_m)(pa, nc, (R)FN(logP)[3], as3);
  FN(m_peq_r_times_m)(qa, nc, (R)FN(logQ)[3], as3);
  FN(m_eq_m_times_m)(as4, nc, as2, as2);
  FN(m_peq_r_times_m)(pa, nc, (R)FN(logP)[4], as4);
  FN(m_peq_r_times_m)(qa, nc, (R)FN(logQ)[4], as4);
  FN(m_eq_m_times_m)(as5, nc, as, as4);
  FN(m_peq_r_times_m)(pa, nc, (R)FN(logP)[5], as5);
  for (int k = 0; k < nc * nc; k++) { qa[k].re += as5[k].re; qa[k].im += as5[k].im; }
  FN(inverse1)(as5, qa, nc);
  FN(m_eq_m_times_m)(qa, nc, pa, as5);
  FN(m_eq_m_times_m)(pa, nc, as3, qa);
  FN(m_peq_r_times_m)(pa, nc, (R)(-0.5), as2);
  for (int k = 0; k < nc * nc; k++) { pa[k].re += as[k].re; pa[k].im += as[k].im; }
  FN(m_eq_r_times_m)(r, nc, (R)16, pa);
  ds = log(ds);
  for (int i = 0; i < nc; i++) EL(r, i, i).re += ds;
}

/* --------------------------------------------- closed forms for nc = 3 */
static FN(mc) FN(cexpi)(R theta)          /* QLA_F_cexpi / QLA_D_cexpi (lib/cmath/QLA_cexpi.c) */
{
  R s, c;
  M_SINCOS(theta, &s, &c);
  FN(mc) z; z.re = c; z.im = s;
  return z;
}

/* x^3 - p2/2 x - det = 0 for the eigenvalues of the traceless Hermitian Q
 * with i Q the input; exp(iQ) = f0 + f1 (iQ) + f2 (iQ)^2
 * (getfs of M_eq_expTA_M.c:139-216, identical in M_eq_expA_M.c) */
static void FN(getfs_exp)(FN(mc) *f0, FN(mc) *f1, FN(mc) *f2, R p2, R det)
{
  R q = (1./6.)*p2;
  R r = -0.5*det;
  R sq = M_SQRT(M_FABS(q));
  R sq3 = sq*sq*sq;
  if (sq3 > M_FABS(r)) {
    R t = M_ACOS(r/sq3);
    FN(mc) sct = FN(cexpi)((1./3.)*t);
    R sqc = sq*sct.re;
    R sqs = 1.73205080756887729352*sq*sct.im;
    R l0 = - 2*sqc;
    R l1 = sqc + sqs;
    R l2 = sqc - sqs;
    R d10 = 0.5*(l1-l0);
    R d20 = 0.5*(l2-l0);
    R d21 = l2-l1;
    FN(mc) eid10, eis01, g10, eid20, eis02, g20, ff0, g2010, b2, f10, z;
    eis01 = FN(cexpi)(0.5*(l0+l1));
    if (d10 == 0) {
      eid10.re = 1; eid10.im = 0.;
      g10 = eis01;
    } else {
      eid10 = FN(cexpi)(d10);
      R sc10 = eid10.im/d10;
      g10.re = sc10*eis01.re; g10.im = sc10*eis01.im;
    }
    ff0.re = eis01.re*eid10.re + eis01.im*eid10.im;   /* eis01 * conj(eid10) */
    ff0.im = eis01.im*eid10.re - eis01.re*eid10.im;
    if (d20 == 0) {
      eid20.re = 1; eid20.im = 0.;
      eis02 = ff0;
      g20 = eis02;
    } else {
      eid20 = FN(cexpi)(d20);
      CMUL(eis02, ff0, eid20);
      R sc20 = eid20.im/d20;
      g20.re = sc20*eis02.re; g20.im = sc20*eis02.im;
    }
    g2010.re = g20.re - g10.re; g2010.im = g20.im - g10.im;
    if (d21 == 0) {
      b2.re = 0; b2.im = 0.;
    } else {
      R d21i = 1/d21;
      b2.re = d21i*g2010.re; b2.im = d21i*g2010.im;
    }
    f2->re = b2.im; f2->im = -b2.re;
    f1->re = (-(l0+l1))*b2.re + g10.re; f1->im = (-(l0+l1))*b2.im + g10.im;
    f10.re = -g10.im; f10.im = g10.re;
    z.re = (l1)*f2->re + f10.re; z.im = (l1)*f2->im + f10.im;
    f0->re = (-l0)*z.re + ff0.re; f0->im = (-l0)*z.im + ff0.im;
  } else {
    if (r == 0) {
      f0->re = 0; f0->im = 0.; f1->re = 0; f1->im = 0.; f2->re = 0; f2->im = 0.;
    } else {
      R a = -M_CBRT(r);
      FN(mc) t, eia, ei3a2, eia2 = FN(cexpi)(0.5*a);
      CMUL(eia, eia2, eia2);
      CMUL(ei3a2, eia, eia2);
      R snc = ei3a2.im/(1.5*a);
      t.re = snc*eia2.re; t.im = snc*eia2.im;
      f1->re = -t.im; f1->im = t.re;
      f2->re = 0; f2->im = 0.;
      t.re = ei3a2.re; t.im = (-1./3.)*ei3a2.im;
      CMUL(*f0, eia2, t);
    }
  }
}

/* M_eq_expTA_M.c:218-274 / M_eq_expA_M.c:222-298 (expA first removes
 * i Im(tr)/3 from the diagonal and multiplies the coefficients by its phase) */
static void FN(exp3_ah)(FN(mc) *e, const FN(mc) *a, int with_trace)
{
  FN(mc) iq[9], mqq[9], f, f0, f1, f2, a0, a1, a2, det0, det1, det2;
  for (int k = 0; k < 9; k++) iq[k] = a[k];
  if (with_trace) {
    R tr = iq[0].im + iq[4].im + iq[8].im;
    R s = (1./3.)*tr;
    iq[0].im = iq[0].im - s;
    iq[4].im = iq[4].im - s;
    iq[8].im = iq[8].im - s;
    f = FN(cexpi)(s);
  }
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      CMUL(mqq[i * 3 + j], iq[i * 3 + 0], iq[0 * 3 + j]);
      CPMS(mqq[i * 3 + j], iq[i * 3 + 1], iq[1 * 3 + j]);
      CPMS(mqq[i * 3 + j], iq[i * 3 + 2], iq[2 * 3 + j]);
    }
  R p2 = -mqq[0].re - mqq[4].re - mqq[8].re;
  R det;
  CMUL(det2, iq[0], iq[4]); CMMS(det2, iq[1], iq[3]);
  CMUL(det1, iq[2], iq[3]); CMMS(det1, iq[0], iq[5]);
  CMUL(det0, iq[1], iq[5]); CMMS(det0, iq[2], iq[4]);
  det = -det2.re*iq[8].im - det2.im*iq[8].re;          /* QLA_r_eqm_Im_c_times_c */
  det -= (det1.re*iq[7].im + det1.im*iq[7].re);        /* QLA_r_meq_Im_c_times_c */
  det -= (det0.re*iq[6].im + det0.im*iq[6].re);
  if (with_trace) {
    FN(getfs_exp)(&f0, &f1, &f2, p2, det);
    CMUL(a0, f, f0);
    CMUL(a1, f, f1);
    CMUL(a2, f, f2);
  } else {
    FN(getfs_exp)(&a0, &a1, &a2, p2, det);
  }
  for (int k = 0; k < 9; k++) {
    CMUL(e[k], a2, mqq[k]);
    CPMS(e[k], a1, iq[k]);
  }
  for (int i = 0; i < 3; i++) { e[i * 4].re += a0.re; e[i * 4].im += a0.im; }
}

/* x^3 - tr x^2 + (tr^2 - p2)/2 x - det = 0 for a positive Hermitian matrix;
 * sqrt (inv = 0) or inverse sqrt (inv = 1) as f0 + f1 m + f2 m^2
 * (getfs of M_eq_sqrtPH_M.c:84-138 and M_eq_invsqrtPH_M.c:84-142) */
static void FN(getfs_sqrtph)(R *f0, R *f1, R *f2, R tr, R p2, R det, int inv)
{
  R tr3 = (1./3.)*tr;
  R p23 = (1./3.)*p2;
  R tr32 = tr3*tr3;
  R q = 0.5*(p23-tr32);
  R r = 0.25*tr3*(5*tr32-p2) - 0.5*det;
  R sq = M_SQRT(M_FABS(q));
  R sq3 = sq*sq*sq;
  if (sq3 > M_FABS(r)) {
    R t = M_ACOS(r/sq3);
    FN(mc) sct = FN(cexpi)((1./3.)*t);
    R sqc = sq*sct.re;
    R sqs = 1.73205080756887729352*sq*sct.im;
    R l0 = tr3 - 2*sqc;
    R ll = tr3 + sqc;
    R l1 = ll + sqs;
    R l2 = ll - sqs;
    R sl0 = M_SQRT(M_FABS(l0));
    R sl1 = M_SQRT(M_FABS(l1));
    R sl2 = M_SQRT(M_FABS(l2));
    R u = sl0 + sl1 + sl2;
    R w = sl0*sl1*sl2;
    if (!inv) {
      R v = sl0*(sl1+sl2) + sl1*sl2;
      R d = (sl0+sl1)*(sl0+sl2)*(sl1+sl2);
      R di = 1./d;
      *f0 = u*w*di;
      *f1 = (tr+v)*di;
      *f2 = -di;
    } else {
      R d = w*(sl0+sl1)*(sl0+sl2)*(sl1+sl2);
      R di = 1./d;
      *f0 = (w*u*u+l0*sl0*(l1+l2)+l1*sl1*(l0+l2)+l2*sl2*(l0+l1))*di;
      *f1 = -(tr*u+w)*di;
      *f2 = u*di;
    }
  } else {
    if (r == 0) {
      *f0 = inv ? 1/M_SQRT(M_FABS(tr3)) : M_SQRT(M_FABS(tr3));
      *f1 = 0;
      *f2 = 0;
    } else {
      R a = -M_CBRT(r);
      R l0 = tr3 + 2*a;
      R l1 = tr3 - a;
      R sl0 = M_SQRT(M_FABS(l0));
      R sl1 = M_SQRT(M_FABS(l1));
      R sl01 = sl0 + sl1;
      if (!inv) {
        *f2 = 0;
        *f1 = (sl01==0) ? 0 : 1/sl01;
        *f0 = sl0*sl1*(*f1);
      } else {
        R p01 = sl0 * sl1;
        R t = p01*sl01;
        R ti = 1/t;
        *f2 = 0;
        *f1 = -ti;
        *f0 = (p01+l0+l1)*ti;
      }
    }
  }
}

/* M_eq_sqrtPH_M.c:140-197 / M_eq_invsqrtPH_M.c:144-201 */
static void FN(sqrtph3)(FN(mc) *fn, const FN(mc) *m, int inv)
{
  FN(mc) mm[9], det0, det1, det2;
  R f0, f1, f2, det;
  R tr = m[0].re + m[4].re + m[8].re;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      CMUL(mm[i * 3 + j], m[i * 3 + 0], m[0 * 3 + j]);
      CPMS(mm[i * 3 + j], m[i * 3 + 1], m[1 * 3 + j]);
      CPMS(mm[i * 3 + j], m[i * 3 + 2], m[2 * 3 + j]);
    }
  R p2 = mm[0].re + mm[4].re + mm[8].re;
  CMUL(det2, m[0], m[4]); CMMS(det2, m[1], m[3]);
  CMUL(det1, m[2], m[3]); CMMS(det1, m[0], m[5]);
  CMUL(det0, m[1], m[5]); CMMS(det0, m[2], m[4]);
  det = det2.re*m[8].re - det2.im*m[8].im;               /* QLA_r_eq_Re_c_times_c */
  det += (det1.re*m[7].re - det1.im*m[7].im);            /* QLA_r_peq_Re_c_times_c */
  det += (det0.re*m[6].re - det0.im*m[6].im);
  FN(getfs_sqrtph)(&f0, &f1, &f2, tr, p2, det, inv);
  for (int k = 0; k < 9; k++) {
    fn[k].re = f2*mm[k].re; fn[k].im = f2*mm[k].im;
    fn[k].re += f1*m[k].re; fn[k].im += f1*m[k].im;
  }
  for (int i = 0; i < 3; i++) fn[i * 4].re += f0;
}

/* eigenvalues of a Hermitian 3x3 matrix (V_eq_eigenvalsH_M.c:106-166) */
static void FN(eigh3)(FN(mc) *v, const FN(mc) *m)
{
  FN(mc) a00 = m[0], a11 = m[4], a22 = m[8], det0, det1, det2;
  R s1, s2, det;
  s1 = (1./3.)*(a00.re + a11.re + a22.re);
  a00.re -= s1;
  a11.re -= s1;
  a22.re -= s1;
  CMUL(det2, a00, a11); CMMS(det2, m[1], m[3]);
  CMUL(det1, m[2], m[3]); CMMS(det1, a00, m[5]);
  CMUL(det0, m[1], m[5]); CMMS(det0, m[2], a11);
  det = det2.re*a22.re - det2.im*a22.im;
  det += (det1.re*m[7].re - det1.im*m[7].im);
  det += (det0.re*m[6].re - det0.im*m[6].im);
  s2 = det2.re;
  s2 += (a00.re*a22.re - a00.im*a22.im);
  s2 -= (m[2].re*m[6].re - m[2].im*m[6].im);
  s2 += (a11.re*a22.re - a11.im*a22.im);
  s2 -= (m[5].re*m[7].re - m[5].im*m[7].im);
  R q = (-1./3.)*s2;
  R r = -0.5*det;
  R sq = M_SQRT(M_FABS(q));
  R sq3 = sq*sq*sq;
  for (int k = 0; k < 3; k++) v[k].im = 0.;
  if (sq3 > M_FABS(r)) {
    R t = M_ACOS(r/sq3);
    FN(mc) sct = FN(cexpi)((1./3.)*t);
    R sqc = sq*sct.re;
    R sqs = 1.73205080756887729352*sq*sct.im;
    R e0 = s1 - 2*sqc;
    R ee = s1 + sqc;
    R e1 = ee + sqs;
    R e2 = ee - sqs;
    v[0].re = e0; v[1].re = e1; v[2].re = e2;
  } else {
    R a = -M_CBRT(r);
    v[0].re = s1 + 2*a;
    v[1].re = s1 - a;
    v[2].re = s1 - a;
  }
}

/* QLA_F_csqrt / QLA_D_csqrt (lib/cmath/QLA_csqrt.c:36-62) */
static FN(mc) FN(csqrt)(FN(mc) z)
{
  R n = M_SQRT(z.re*z.re + z.im*z.im);
  R r = z.re;
  R i = z.im;
  R sr = M_SQRT(M_FABS(0.5*(n+r)));
  R si = M_COPYSIGN(M_SQRT(M_FABS(0.5*(n-r))), i);
  FN(mc) c; c.re = sr; c.im = si;
  return c;
}

/* QLA_F_cpow / QLA_D_cpow (lib/cmath/QLA_cpow.c:36-58) */
static FN(mc) FN(cpow)(FN(mc) a, R b)
{
  R r = pow(a.re*a.re + a.im*a.im, 0.5*b);
  R theta = b*M_ATAN2(a.im, a.re);
  FN(mc) c = FN(cexpi)(theta);
  c.re = r*c.re; c.im = r*c.im;
  return c;
}

/* eigenvalues of a general complex 3x3 matrix via the depressed cubic
 * (V_eq_eigenvals_M.c:127-186, the branch the template compiles) */
static void FN(eig3)(FN(mc) *v, const FN(mc) *m)
{
  FN(mc) a00 = m[0], a11 = m[4], a22 = m[8], s1, s2, det0, det1, det2, det;
  s1.re = a00.re + a11.re; s1.im = a00.im + a11.im;
  s1.re += a22.re; s1.im += a22.im;
  s1.re = (1./3.)*s1.re; s1.im = (1./3.)*s1.im;
  a00.re -= s1.re; a00.im -= s1.im;
  a11.re -= s1.re; a11.im -= s1.im;
  a22.re -= s1.re; a22.im -= s1.im;
  CMUL(det2, a00, a11); CMMS(det2, m[1], m[3]);
  CMUL(det1, m[2], m[3]); CMMS(det1, a00, m[5]);
  CMUL(det0, m[1], m[5]); CMMS(det0, m[2], a11);
  CMUL(det, det2, a22);
  CPMS(det, det1, m[7]);
  CPMS(det, det0, m[6]);
  s2 = det2;
  CPMS(s2, a00, a22);
  CMMS(s2, m[2], m[6]);
  CPMS(s2, a11, a22);
  CMMS(s2, m[5], m[7]);
  FN(mc) p, q, p2, q2, t, d, w0, w, pw0, e0, e1, e2;
  p.re = (1./3.)*s2.re; p.im = (1./3.)*s2.im;
  q.re = (-0.5)*det.re; q.im = (-0.5)*det.im;
  CMUL(p2, p, p);
  CMUL(q2, q, q);
  d.re = p.re*p2.re - p.im*p2.im + q2.re;                /* QLA_c_eq_c_times_c_plus_c */
  d.im = p.re*p2.im + p.im*p2.re + q2.im;
  t = FN(csqrt)(d);
  R ts = q.re*t.re + q.im*t.im;                         /* QLA_r_eq_Re_ca_times_c */
  if (ts >= 0) { q.re += t.re; q.im += t.im; }
  else { q.re -= t.re; q.im -= t.im; }
  w0 = FN(cpow)(q, 1./3.);
  w.re = -0.5; w.im = 0.86602540378443864676;
  {                                                    /* safedivC(&pw0, &p, &w0, 0) */
    R dd = w0.re*w0.re + w0.im*w0.im;
    if (dd == 0) {
      pw0.re = 0; pw0.im = 0.;
    } else {
      R di = 1/dd;
      pw0.re = p.re*w0.re + p.im*w0.im;
      pw0.im = p.im*w0.re - p.re*w0.im;
      pw0.re = di*pw0.re; pw0.im = di*pw0.im;
    }
  }
  e0.re = pw0.re - w0.re; e0.im = pw0.im - w0.im;
  v[0].re = s1.re + e0.re; v[0].im = s1.im + e0.im;
  e1.re = w.re*pw0.re + w.im*pw0.im;                   /* conj(w) * pw0 */
  e1.im = w.re*pw0.im - w.im*pw0.re;
  CMMS(e1, w, w0);
  v[1].re = s1.re + e1.re; v[1].im = s1.im + e1.im;
  CMUL(e2, w, pw0);
  e2.re -= w.re*w0.re + w.im*w0.im;                    /* -= conj(w) * w0 */
  e2.im -= w.re*w0.im - w.im*w0.re;
  v[2].re = s1.re + e2.re; v[2].im = s1.im + e2.im;
}

/* ------------------------------------------- eigenvalues, nc > 3 (QR) */
/* 2x2 eigenvalues used when the QR iteration deflates a 2x2 block: the
 * Hermitian form (V_eq_eigenvalsH_M.c:82-104) and the general complex form
 * (V_eq_eigenvals_M.c:82-125, the "more accurate" branch) */
static void FN(eig2_h)(FN(mc) *v0, FN(mc) *v1, const FN(mc) *m00, const FN(mc) *m01, const FN(mc) *m10,
                       const FN(mc) *m11)
{
  R tr, det;
  det = m00->re*m11->re - m00->im*m11->im;
  det -= (m01->re*m10->re - m01->im*m10->im);
  tr = m00->re + m11->re;
  if (det == 0) {
    v0->re = 0; v0->im = 0.;
    v1->re = tr; v1->im = 0.;
  } else {
    R ss = 0.5*tr;
    R d = ss*ss - det;
    R sd = M_SQRT(M_FABS(d));
    R l0, l1 = ss + M_COPYSIGN(sd, ss);
    l0 = det / l1;
    v0->re = l0; v0->im = 0.;
    v1->re = l1; v1->im = 0.;
  }
}

static void FN(cdiv)(FN(mc) *c, FN(mc) a, FN(mc) b)    /* QLA_c_eq_c_div_c */
{
  R t = 1.0/(b.re*b.re + b.im*b.im);
  c->re = (a.re*b.re + a.im*b.im)*t;
  c->im = (a.im*b.re - a.re*b.im)*t;
}

static void FN(eig2_g)(FN(mc) *v0, FN(mc) *v1, const FN(mc) *m00, const FN(mc) *m01, const FN(mc) *m10,
                       const FN(mc) *m11)
{
  FN(mc) tr, det;
  CMUL(det, *m00, *m11);
  CMMS(det, *m01, *m10);
  tr.re = m00->re + m11->re; tr.im = m00->im + m11->im;
  if (det.re == 0 && det.im == 0) {
    v0->re = 0; v0->im = 0.;
    *v1 = tr;
  } else {
    FN(mc) ss, d, sd;
    ss.re = 0.5*tr.re; ss.im = 0.5*tr.im;
    CMUL(d, ss, ss);
    d.re -= det.re; d.im -= det.im;
    sd = FN(csqrt)(d);
    R ts = ss.re*sd.re + ss.im*sd.im;
    if (ts >= 0) { v1->re = ss.re + sd.re; v1->im = ss.im + sd.im; }
    else { v1->re = ss.re - sd.re; v1->im = ss.im - sd.im; }
    FN(cdiv)(v0, det, *v1);
  }
}

/* Hessenberg reduction with pivoting through a row/column permutation
 * (V_eq_eigenvalsH_M.c:195-245, identical in V_eq_eigenvals_M.c), then the
 * implicit double-shift QR iteration (V_eq_eigenvalsH_M.c:315-483).  The
 * template's iteration has no overall bound (after 100 iterations on one
 * eigenvalue it writes the diagonal and starts over); here a search for one
 * eigenvalue gives up after ORA_QR_MAXITS restarts, leaving that diagonal. */
#define ORA_QR_MAXITS 20
static void FN(eig_qr)(FN(mc) *v, const FN(mc) *a, int nc, int herm)
{
  FN(mc) mm[ORA_NCMAX * ORA_NCMAX], h[ORA_NCMAX * ORA_NCMAX];
  int rc[ORA_NCMAX];
  for (int i = 0; i < nc; i++) {
    for (int j = 0; j < nc; j++) mm[i * nc + j] = a[i * nc + j];
    rc[i] = i;
  }
#define MP(i, j) mm[rc[i] * nc + rc[j]]
  for (int k = 0; k < nc - 2; k++) {
    FN(mc) sk;
    R rmax = MP(k + 1, k).re*MP(k + 1, k).re + MP(k + 1, k).im*MP(k + 1, k).im;
    int imax = k + 1;
    for (int i = k + 2; i < nc; i++) {
      R n2 = MP(i, k).re*MP(i, k).re + MP(i, k).im*MP(i, k).im;
      if (n2 > rmax) { rmax = n2; imax = i; }
    }
    if (rmax == 0) continue;
    { int rk = rc[k + 1]; rc[k + 1] = rc[imax]; rc[imax] = rk; }
    rmax = 1/rmax;
    sk.re = rmax*MP(k + 1, k).re; sk.im = -(rmax*MP(k + 1, k).im);   /* QLA_c_eq_r_times_ca */
    for (int i = k + 2; i < nc; i++) {
      FN(mc) t;
      CMUL(t, sk, MP(i, k));
      MP(i, k).re = 0; MP(i, k).im = 0.;
      for (int j = k + 1; j < nc; j++) CMMS(MP(i, j), t, MP(k + 1, j));
      for (int j = 0; j < nc; j++) CPMS(MP(j, k + 1), t, MP(j, i));
    }
  }
  for (int i = 0; i < nc; i++)
    for (int j = 0; j < nc; j++) h[i * nc + j] = MP(i, j);
#undef MP
#define MH(i, j) h[(i) * nc + (j)]
#define CABS(z) M_SQRT((z).re*(z).re + (z).im*(z).im)
#define CNORM2(z) ((z).re*(z).re + (z).im*(z).im)
  R anorm = 0;
  for (int i = 0; i < nc; i++)
    for (int j = (i == 0 ? 0 : i - 1); j < nc; j++) anorm += CABS(MH(i, j));
  int nn = nc - 1, restarts = 0;
  FN(mc) t; t.re = 0; t.im = 0.;
  while (nn >= 0) {
    int l, its = 0;
    do {
      for (l = nn; l > 0; l--) {
        R s = CABS(MH(l - 1, l - 1)) + CABS(MH(l, l));
        if (s == 0) s = anorm;
        R o = CABS(MH(l, l - 1));
        if (s + o == s) { MH(l, l - 1).re = 0; MH(l, l - 1).im = 0.; break; }
      }
      FN(mc) x = MH(nn, nn);
      if (l == nn) {
        v[nn].re = x.re + t.re; v[nn].im = x.im + t.im;
        nn--;
      } else if (l == nn - 1) {
        if (herm) FN(eig2_h)(&v[nn - 1], &v[nn], &MH(nn - 1, nn - 1), &MH(nn - 1, nn), &MH(nn, nn - 1), &x);
        else FN(eig2_g)(&v[nn - 1], &v[nn], &MH(nn - 1, nn - 1), &MH(nn - 1, nn), &MH(nn, nn - 1), &x);
        v[nn - 1].re += t.re; v[nn - 1].im += t.im;
        v[nn].re += t.re; v[nn].im += t.im;
        nn -= 2;
      } else {
        if (its >= 100) {
          for (int i = 0; i <= nn; i++) { v[i].re = MH(i, i).re + t.re; v[i].im = MH(i, i).im + t.im; }
          break;
        }
        FN(mc) y, w, p, q, r;
        y = MH(nn - 1, nn - 1);
        CMUL(w, MH(nn, nn - 1), MH(nn - 1, nn));
        if (its == 10 || its == 20) {
          t.re += x.re; t.im += x.im;
          for (int i = 0; i < nn; i++) { MH(i, i).re -= x.re; MH(i, i).im -= x.im; }
          MH(nn, nn).re = 0; MH(nn, nn).im = 0.;
          x.re = 0; x.im = 0.;
          y = MH(nn - 1, nn - 1);
          R s = CABS(MH(nn, nn - 1)) + CABS(MH(nn - 1, nn - 2));
          x.re = 0.75*s; x.im = 0.;
          y = x;
          w.re = -0.4375*s*s; w.im = 0.;
        }
        its++;
        int m = l;
        {
          FN(mc) rr, ss, t1, z = MH(m, m);
          rr.re = x.re - z.re; rr.im = x.im - z.im;
          ss.re = y.re - z.re; ss.im = y.im - z.im;
          CMUL(p, rr, ss);
          p.re -= w.re; p.im -= w.im;
          CPMS(p, MH(m + 1, m), MH(m, m + 1));
          t1.re = MH(m + 1, m + 1).re - z.re; t1.im = MH(m + 1, m + 1).im - z.im;
          t1.re -= rr.re + ss.re; t1.im -= rr.im + ss.im;
          CMUL(q, MH(m + 1, m), t1);
          CMUL(r, MH(m + 1, m), MH(m + 2, m + 1));
        }
        for (int k = m; k < nn; k++) {
          R xx = 0;
          if (k != m) {
            p = MH(k, k - 1);
            q = MH(k + 1, k - 1);
            r.re = 0; r.im = 0.;
            if (k + 1 != nn) r = MH(k + 2, k - 1);
            xx = CABS(p) + CABS(q) + CABS(r);
            if (xx != 0) {
              R xxi = 1/xx;
              p.re = xxi*p.re; p.im = xxi*p.im;
              q.re = xxi*q.re; q.im = xxi*q.im;
              r.re = xxi*r.re; r.im = xxi*r.im;
            }
          }
          R p2 = CNORM2(p);
          R s2 = p2 + CNORM2(q) + CNORM2(r);
          if (s2 != 0) {
            FN(mc) sv, t1;
            if (p2 > 0) { sv.re = (sqrt(s2/p2))*p.re; sv.im = (sqrt(s2/p2))*p.im; }
            else { sv.re = sqrt(s2); sv.im = 0.; }
            if (k == m) {
              if (l != m) { MH(k, k - 1).re = -MH(k, k - 1).re; MH(k, k - 1).im = -MH(k, k - 1).im; }
            } else {
              MH(k, k - 1).re = (-xx)*sv.re; MH(k, k - 1).im = (-xx)*sv.im;
              MH(k + 1, k - 1).re = 0; MH(k + 1, k - 1).im = 0.;
              if (k + 2 < nc) { MH(k + 2, k - 1).re = 0; MH(k + 2, k - 1).im = 0.; }
            }
            p.re += sv.re; p.im += sv.im;
            FN(cdiv)(&x, p, sv);
            FN(cdiv)(&y, q, sv);
            FN(cdiv)(&w, r, sv);
            FN(cdiv)(&t1, q, p); q = t1;
            FN(cdiv)(&t1, r, p); r = t1;
            for (int j = k; j <= nn; j++) {
              p = MH(k, j);
              p.re += q.re*MH(k + 1, j).re + q.im*MH(k + 1, j).im;   /* += conj(q) M */
              p.im += q.re*MH(k + 1, j).im - q.im*MH(k + 1, j).re;
              if (k + 1 != nn) {
                p.re += r.re*MH(k + 2, j).re + r.im*MH(k + 2, j).im;
                p.im += r.re*MH(k + 2, j).im - r.im*MH(k + 2, j).re;
                CMMS(MH(k + 2, j), p, w);
              }
              CMMS(MH(k + 1, j), p, y);
              CMMS(MH(k, j), p, x);
            }
            for (int i = l; i <= (nn < k + 3 ? nn : k + 3); i++) {
              CMUL(p, x, MH(i, k));
              CPMS(p, y, MH(i, k + 1));
              if (k + 1 != nn) {
                CPMS(p, w, MH(i, k + 2));
                MH(i, k + 2).re -= p.re*r.re + p.im*r.im;             /* -= p conj(r) */
                MH(i, k + 2).im -= p.im*r.re - p.re*r.im;
              }
              MH(i, k + 1).re -= p.re*q.re + p.im*q.im;
              MH(i, k + 1).im -= p.im*q.re - p.re*q.im;
              MH(i, k).re -= p.re; MH(i, k).im -= p.im;
            }
          }
        }
      }
    } while (l + 1 < nn);
    if (its >= 100 && ++restarts >= ORA_QR_MAXITS) break;
  }
#undef MH
#undef CABS
#undef CNORM2
}

/* --------------------------------------------- closed forms for nc = 2 */
/* The templates' `if(NC==2)` branches, compiled into the two-colour
 * libraries and taken by the N-colour libraries at nc = 2.  Each operation
 * restates the complex macro the template calls (include/qla_complex.h):
 * QLA_c_eq_r_div_c t = a / |b|^2 in R; QLA_c_eq_c_div_c t = 1.0 / |b|^2 in
 * double, rounded; QLA_c_eq_c_times_c_plus_c left to right. */

/* QLA_F_cexp / QLA_D_cexp (lib/cmath/QLA_cexp.c, the compiled branch) */
static FN(mc) FN(cexp)(FN(mc) a)
{
  R mag = M_EXP(a.re);
  R s, c;
  M_SINCOS(a.im, &s, &c);
  FN(mc) z; z.re = mag*c; z.im = mag*s;
  return z;
}

/* QLA_F_clog / QLA_D_clog (lib/cmath/QLA_clog.c): log in double */
static FN(mc) FN(clog)(FN(mc) a)
{
  FN(mc) z;
  z.re = 0.5*log(a.re*a.re + a.im*a.im);
  z.im = M_ATAN2(a.im, a.re);
  return z;
}

/* QLA_F_csinhcosh / QLA_D_csinhcosh (lib/cmath/QLA_csinhcosh.c, the
 * compiled branch: cosh x = sqrt(1 + sinh^2 x)) */
static void FN(csinhcosh)(FN(mc) a, FN(mc) *sh, FN(mc) *ch)
{
  R sx = M_SINH(a.re);
  R cx = M_SQRT(1+sx*sx);
  R sy, cy;
  M_SINCOS(a.im, &sy, &cy);
  sh->re = cy*sx; sh->im = sy*cx;
  ch->re = cy*cx; ch->im = sy*sx;
}

static void FN(rdivc)(FN(mc) *c, int a, FN(mc) b)     /* QLA_c_eq_r_div_c, a integer */
{
  R t = a/(b.re*b.re + b.im*b.im);
  c->re = t*b.re;
  c->im = -t*b.im;
}

#define CTCPC(r, p, x, q) { (r).re = (p).re*(x).re - (p).im*(x).im + (q).re; \
                            (r).im = (p).re*(x).im + (p).im*(x).re + (q).im; }
#define CEQM(r, p, q) { (r).re = -(p).re*(q).re + (p).im*(q).im; (r).im = -(p).re*(q).im - (p).im*(q).re; }
/* r = c0 + c1 a for complex c0, c1 */
#define OUT_C(r, c0, c1, a00, a01, a10, a11) { CTCPC(r[0], c1, a00, c0); CMUL(r[1], c1, a01); \
                                              CMUL(r[2], c1, a10); CTCPC(r[3], c1, a11, c0); }
/* r = c0 + c1 a for real c0, c1 (QLA_c_eq_c_times_r_plus_r, QLA_c_eq_c_times_r) */
#define OUT_R(r, c0, c1, a00, a01, a10, a11) { \
    r[0].re = a00.re*(c1) + (c0); r[0].im = a00.im*(c1); \
    r[1].re = (c1)*a01.re; r[1].im = (c1)*a01.im; \
    r[2].re = (c1)*a10.re; r[2].im = (c1)*a10.im; \
    r[3].re = a11.re*(c1) + (c0); r[3].im = a11.im*(c1); }

/* M_eq_exp_M.c:257-291 */
static void FN(exp2)(FN(mc) *r, const FN(mc) *a)
{
  FN(mc) a00 = a[0], a01 = a[1], a10 = a[2], a11 = a[3], tr, s, mdet, t, st, ch, c0, c1, es;
  tr.re = a00.re + a11.re; tr.im = a00.im + a11.im;
  s.re = 0.5*tr.re; s.im = 0.5*tr.im;
  a00.re -= s.re; a00.im -= s.im;
  a11.re -= s.re; a11.im -= s.im;
  CMUL(mdet, a01, a10);
  CMMS(mdet, a00, a11);
  t = FN(csqrt)(mdet);
  if (t.re == 0 && t.im == 0) {
    st.re = 1; st.im = 0;
    ch.re = 1; ch.im = 0;
  } else {
    FN(mc) sh;
    FN(csinhcosh)(t, &sh, &ch);
    FN(cdiv)(&st, sh, t);
  }
  es = FN(cexp)(s);
  CMUL(c0, es, ch);
  CMUL(c1, es, st);
  OUT_C(r, c0, c1, a00, a01, a10, a11);
}

/* eigenvalues l0, l1 of a 2x2 matrix, as M_eq_sqrt_M.c:94-115 and
 * M_eq_invsqrt_M.c:95-116 compute them (the eig2_g arithmetic) */
static void FN(sqrt2_common)(FN(mc) *r, const FN(mc) *a, int inv)
{
  FN(mc) l0, l1, sl0, sl1, ss, ps, c0, c1, tr;
  FN(eig2_g)(&l0, &l1, &a[0], &a[1], &a[2], &a[3]);
  tr.re = a[0].re + a[3].re; tr.im = a[0].im + a[3].im;
  sl0 = FN(csqrt)(l0);
  sl1 = FN(csqrt)(l1);
  ss.re = sl0.re + sl1.re; ss.im = sl0.im + sl1.im;
  CMUL(ps, sl0, sl1);
  if (!inv) {                                  /* M_eq_sqrt_M.c:116-132 */
    if (ss.re == 0 && ss.im == 0) {
      c0 = sl0;
      c1.re = 0; c1.im = 0;
    } else {
      FN(rdivc)(&c1, 1, ss);
      CMUL(c0, ps, c1);
    }
  } else {                                     /* M_eq_invsqrt_M.c:117-131 */
    FN(mc) t;
    CMUL(t, ps, ss);
    FN(rdivc)(&c1, -1, t);
    ps.re += tr.re; ps.im += tr.im;
    CEQM(c0, ps, c1);
  }
  OUT_C(r, c0, c1, a[0], a[1], a[2], a[3]);
}

/* M_eq_log_M.c:103-152 */
static void FN(log2)(FN(mc) *r, const FN(mc) *a)
{
  FN(mc) tr, s, det, d, c0, c1;
  tr.re = a[0].re + a[3].re; tr.im = a[0].im + a[3].im;
  s.re = 0.5*tr.re; s.im = 0.5*tr.im;
  CMUL(det, a[0], a[3]);
  CMMS(det, a[1], a[2]);
  CMUL(d, s, s);
  d.re -= det.re; d.im -= det.im;
  if (d.re == 0 && d.im == 0) {
    FN(mc) ls = FN(clog)(s);
    c0.re = 0; c0.im = 0;
    FN(cdiv)(&c1, ls, s);
  } else {
    FN(mc) e0, e1, de, sd = FN(csqrt)(d), le0, le1, dei, dl, dl0;
    R ts = s.re*sd.re + s.im*sd.im;
    if (ts >= 0) {
      e1.re = s.re + sd.re; e1.im = s.im + sd.im;
      de.re = 2*sd.re; de.im = 2*sd.im;
    } else {
      e1.re = s.re - sd.re; e1.im = s.im - sd.im;
      de.re = -2*sd.re; de.im = -2*sd.im;
    }
    FN(cdiv)(&e0, det, e1);
    le0 = FN(clog)(e0);
    le1 = FN(clog)(e1);
    FN(rdivc)(&dei, 1, de);
    dl.re = le1.re - le0.re; dl.im = le1.im - le0.im;
    CMUL(dl0, e1, le0);
    CMMS(dl0, e0, le1);
    CMUL(c1, dl, dei);
    CMUL(c0, dl0, dei);
  }
  OUT_C(r, c0, c1, a[0], a[1], a[2], a[3]);
}

/* M_eq_expA_M.c:312-350 (with_trace) and M_eq_expTA_M.c:301-329 */
static void FN(expah2)(FN(mc) *r, const FN(mc) *a, int with_trace)
{
  FN(mc) a00 = a[0], a01 = a[1], a10 = a[2], a11 = a[3];
  R det, t;
  if (with_trace) {
    FN(mc) tr, s, sc, c0, c1, es;
    R st, cs;
    tr.re = a00.re + a11.re; tr.im = a00.im + a11.im;
    s.re = 0.5*tr.re; s.im = 0.5*tr.im;
    a00.re -= s.re; a00.im -= s.im;
    a11.re -= s.re; a11.im -= s.im;
    det = a00.re*a11.re - a00.im*a11.im;
    det -= (a01.re*a10.re - a01.im*a10.im);
    t = M_SQRT(M_FABS(det));
    if (t == 0) {
      st = 1;
      cs = 1;
    } else {
      sc = FN(cexpi)(t);
      st = sc.im/t;
      cs = sc.re;
    }
    es = FN(cexpi)(s.im);
    c0.re = cs*es.re; c0.im = cs*es.im;
    c1.re = st*es.re; c1.im = st*es.im;
    OUT_C(r, c0, c1, a00, a01, a10, a11);
  } else {
    R c0, c1;
    det = a00.re*a11.re - a00.im*a11.im;
    det -= (a01.re*a10.re - a01.im*a10.im);
    t = M_SQRT(M_FABS(det));
    if (t == 0) {
      c0 = 1;
      c1 = 1;
    } else {
      FN(mc) sc = FN(cexpi)(t);
      c0 = sc.re;
      c1 = sc.im/t;
    }
    OUT_R(r, c0, c1, a00, a01, a10, a11);
  }
}

/* M_eq_sqrtPH_M.c:224-262 (inv = 0) and M_eq_invsqrtPH_M.c:228-251 */
static void FN(sqrtph2)(FN(mc) *r, const FN(mc) *a, int inv)
{
  const FN(mc) a00 = a[0], a01 = a[1], a10 = a[2], a11 = a[3];
  R tr, det, sdet, c0, c1;
  det = a00.re*a11.re - a00.im*a11.im;
  det -= (a01.re*a10.re - a01.im*a10.im);
  tr = a00.re + a11.re;
  if (inv) {
    sdet = M_SQRT(M_FABS(det));
    c1 = 1/(sdet*M_SQRT(M_FABS(tr+2*sdet)));
    c0 = (tr+sdet)*c1;
    c1 = -c1;
    OUT_R(r, c0, c1, a00, a01, a10, a11);
  } else if (det == 0) {
    if (tr == 0) {
      for (int k = 0; k < 4; k++) { r[k].re = 0; r[k].im = 0; }
    } else {
      c1 = 1/M_SQRT(M_FABS(tr));
      r[0].re = c1*a00.re; r[0].im = c1*a00.im;
      r[1].re = c1*a01.re; r[1].im = c1*a01.im;
      r[2].re = c1*a10.re; r[2].im = c1*a10.im;
      r[3].re = c1*a11.re; r[3].im = c1*a11.im;
    }
  } else {
    sdet = M_SQRT(M_FABS(det));
    c1 = 1/M_SQRT(M_FABS(tr+2*sdet));
    c0 = sdet*c1;
    OUT_R(r, c0, c1, a00, a01, a10, a11);
  }
}

/* C_eq_det_M.c:63-69, M_eq_inverse_M.c:64-78 */
static void FN(det2)(FN(mc) *det, const FN(mc) *a)
{
  CMUL(*det, a[0], a[3]);
  CMMS(*det, a[1], a[2]);
}

static void FN(inverse2)(FN(mc) *x, const FN(mc) *a)
{
  FN(mc) det, idet;
  FN(det2)(&det, a);
  FN(rdivc)(&idet, 1, det);
  CMUL(x[0], a[3], idet);
  CEQM(x[1], a[1], idet);
  CEQM(x[2], a[2], idet);
  CMUL(x[3], a[0], idet);
}

/* V_eq_M_inverse_V.c:65-83 (nb = 1), M_eq_M_inverse_M.c:65-91 (nb = 2) */
static void FN(minv2)(FN(mc) *x, const FN(mc) *a, const FN(mc) *b, int nb)
{
  FN(mc) det, idet, rr[4];
  FN(det2)(&det, a);
  FN(rdivc)(&idet, 1, det);
  for (int j = 0; j < nb; j++) {
    CMUL(rr[j], a[3], b[j]);
    CMMS(rr[j], a[1], b[nb + j]);
    CMUL(rr[nb + j], a[0], b[nb + j]);
    CMMS(rr[nb + j], a[2], b[j]);
  }
  for (int k = 0; k < 2 * nb; k++) CMUL(x[k], rr[k], idet);
}
#undef CTCPC
#undef CEQM
#undef OUT_C
#undef OUT_R

/* x = a^-1 b for b with nb columns (a ColorVector: nb = 1; a ColorMatrix:
 * nb = nc): V_eq_M_inverse_V.c:84-126 for nc = 3 and nb = 1 (Cramer's
 * rule), else Gauss-Jordan (V_eq_M_inverse_V.c:128-168, M_eq_M_inverse_M.c:85-135) */
static void FN(minv1)(FN(mc) *x, const FN(mc) *a, const FN(mc) *b, int nc, int nb)
{
  if (nc == 2) {
    FN(minv2)(x, a, b, nb);
    return;
  }
  if (nc == 3 && nb == 1) {
    FN(mc) det0, det1, det2, det, idet, r0, r1, r2;
    CMUL(det2, a[0], a[4]); CMMS(det2, a[1], a[3]);
    CMUL(det1, a[2], a[3]); CMMS(det1, a[0], a[5]);
    CMUL(det0, a[1], a[5]); CMMS(det0, a[2], a[4]);
    CMUL(det, det2, a[8]);
    CPMS(det, det1, a[7]);
    CPMS(det, det0, a[6]);
    {
      R t = 1 / (det.re * det.re + det.im * det.im);
      idet.re = t * det.re;
      idet.im = -t * det.im;
    }
#define SETV(rr, j0, i1, j1, i2, j2) \
    CMUL(det, a[i1 * 3 + j1], a[i2 * 3 + j2]); CMMS(det, a[i1 * 3 + j2], a[i2 * 3 + j1]); CPMS(rr, det, b[j0]);
    CMUL(r0, det0, b[2]);
    SETV(r0, 0, 1, 1, 2, 2);
    SETV(r0, 1, 2, 1, 0, 2);
    CMUL(r1, det1, b[2]);
    SETV(r1, 0, 1, 2, 2, 0);
    SETV(r1, 1, 2, 2, 0, 0);
    CMUL(r2, det2, b[2]);
    SETV(r2, 0, 1, 0, 2, 1);
    SETV(r2, 1, 2, 0, 0, 1);
#undef SETV
    CMUL(x[0], r0, idet);
    CMUL(x[1], r1, idet);
    CMUL(x[2], r2, idet);
    return;
  }
  FN(m_eq_m_inverse_m)(x, nc, a, b, nb);
}

/* ------------------------------------------------------------ v-forms */
/* r[i] = f(a[i]); eigenvalue functions write nc complex numbers per site,
 * det one.  nc = 2 takes the templates' two-colour closed forms; the
 * closed nc = 3 forms exist only for nc == 3; other colour counts take the templates' generic paths (expA / expTA: the exp path;
 * sqrtPH / invsqrtPH: the Newton paths; eigenvalues: Hessenberg + QR). */
int FN(ora_mfunc)(R *r, const R *a, long n, int nc, int which)
{
  const FN(mc) *A = (const FN(mc) *)a;
  FN(mc) *O = (FN(mc) *)r;
  const double eps = sizeof(R) == 4 ? (double)FLT_EPSILON : DBL_EPSILON;
  for (long i = 0; i < n; i++) {
    const FN(mc) *ai = A + i * nc * nc;
    FN(mc) *oi = O + i * nc * nc;
    if (nc == 2) {
      switch (which) {
      case ORA_MF_EXP: FN(exp2)(oi, ai); break;
      case ORA_MF_SQRT: FN(sqrt2_common)(oi, ai, 0); break;
      case ORA_MF_INVERSE: FN(inverse2)(oi, ai); break;
      case ORA_MF_DET: FN(det2)(O + i, ai); break;
      case ORA_MF_INVSQRT: FN(sqrt2_common)(oi, ai, 1); break;
      case ORA_MF_LOG: FN(log2)(oi, ai); break;
      case ORA_MF_EXPA: FN(expah2)(oi, ai, 1); break;
      case ORA_MF_EXPTA: FN(expah2)(oi, ai, 0); break;
      case ORA_MF_SQRTPH: FN(sqrtph2)(oi, ai, 0); break;
      case ORA_MF_INVSQRTPH: FN(sqrtph2)(oi, ai, 1); break;
      case ORA_MF_EIGENVALS: FN(eig2_g)(O + i * 2, O + i * 2 + 1, ai, ai + 1, ai + 2, ai + 3); break;
      case ORA_MF_EIGENVALSH: FN(eig2_h)(O + i * 2, O + i * 2 + 1, ai, ai + 1, ai + 2, ai + 3); break;
      default: return -1;
      }
      continue;
    }
    switch (which) {
    case ORA_MF_EXP: FN(exp1)(oi, ai, nc); break;
    case ORA_MF_SQRT: FN(sqrt1)(oi, ai, nc, eps); break;
    case ORA_MF_INVERSE: FN(inverse1)(oi, ai, nc); break;
    case ORA_MF_DET: FN(det1)(O + i, ai, nc); break;
    case ORA_MF_INVSQRT: FN(invsqrt1)(oi, ai, nc, eps); break;
    case ORA_MF_LOG: FN(log1)(oi, ai, nc, eps); break;
    case ORA_MF_EXPA:
      if (nc == 3) FN(exp3_ah)(oi, ai, 1); else FN(exp1)(oi, ai, nc);
      break;
    case ORA_MF_EXPTA:
      if (nc == 3) FN(exp3_ah)(oi, ai, 0); else FN(exp1)(oi, ai, nc);
      break;
    case ORA_MF_SQRTPH:
      if (nc == 3) FN(sqrtph3)(oi, ai, 0); else FN(sqrt1)(oi, ai, nc, eps);
      break;
    case ORA_MF_INVSQRTPH:
      if (nc == 3) FN(sqrtph3)(oi, ai, 1); else FN(invsqrt1)(oi, ai, nc, eps);
      break;
    case ORA_MF_EIGENVALS:
      if (nc == 3) FN(eig3)(O + i * 3, ai); else FN(eig_qr)(O + i * nc, ai, nc, 0);
      break;
    case ORA_MF_EIGENVALSH:
      if (nc == 3) FN(eigh3)(O + i * 3, ai); else FN(eig_qr)(O + i * nc, ai, nc, 1);
      break;
    default: return -1;
    }
  }
  return 0;
}

/* r[i] = a[ia[i]]^-1 b[ib[i]] (index arrays may be NULL); b, r hold nb
 * columns per site (1: ColorVector, nc: ColorMatrix) */
void FN(ora_minv)(R *r, const R *a, const R *b, long n, int nc, int nb, const int *ia, const int *ib)
{
  const FN(mc) *A = (const FN(mc) *)a, *B = (const FN(mc) *)b;
  FN(mc) *O = (FN(mc) *)r;
  for (long i = 0; i < n; i++) {
    const long ja = ia ? ia[i] : i, jb = ib ? ib[i] : i;
    FN(minv1)(O + i * nc * nb, A + ja * nc * nc, B + jb * nc * nb, nc, nb);
  }
}

#undef CMUL
#undef CMMS
#undef CPMS
#undef EL
#undef FN
#undef CAT2
#undef CAT2_
