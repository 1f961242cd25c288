/*
 * Test infrastructure (the oracle): restatement of QLA's matrix-function code
 * templates (the C files under lib/perl/code-templates), precision-generic.  Included twice
 * by qla_oracle_mfunc.c with R = float / double and SFX = f / d, mirroring the
 * reference's F and D builds of the same templates.  nc is a run-time colour
 * count (<= ORA_NCMAX), as in the reference's N-colour build; for nc == 3 the
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
static void FN(m_eq_m_inverse_m)(FN(mc) *x, int nc, const FN(mc) *a, const FN(mc) *b)
{
  FN(mc) c[ORA_NCMAX * ORA_NCMAX], d[ORA_NCMAX * ORA_NCMAX];
  int row[ORA_NCMAX];
  for (int i = 0; i < nc; i++) {
    for (int j = 0; j < nc; j++) { EL(c, i, j) = EL(a, i, j); EL(d, i, j) = EL(b, i, j); }
    row[i] = i;
  }
#define CC(i, j) EL(c, row[i], j)
#define DD(i, j) EL(d, row[i], j)
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
      for (int j = 0; j < nc; j++) {
        DD(i, j).re -= (t.re * DD(k, j).re - t.im * DD(k, j).im);
        DD(i, j).im -= (t.re * DD(k, j).im + t.im * DD(k, j).re);
      }
    }
  }
  for (int i = 0; i < nc; i++)
    for (int j = 0; j < nc; j++) {
      FN(mc) u = CC(i, i), v = DD(i, j);
      EL(x, i, j).re = u.re * v.re - u.im * v.im;
      EL(x, i, j).im = u.re * v.im + u.im * v.re;
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
  FN(mc) one[ORA_NCMAX * ORA_NCMAX];
  FN(m_eq_d)(one, nc, 1);
  FN(m_eq_m_inverse_m)(x, nc, a, one);
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
  FN(m_eq_m_inverse_m)(qb, nc, pb, bs6);
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
static void FN(sqrt1)(FN(mc) *r, const FN(mc) *a, int nc, double eps)
{
  double ds = FN(fnorm2)(a, nc);
  if (ds == 0) { FN(m_eq_d)(r, nc, 0); return; }
  ds = sqrt(ds);
  FN(mc) x[ORA_NCMAX * ORA_NCMAX], e[ORA_NCMAX * ORA_NCMAX], t1[ORA_NCMAX * ORA_NCMAX],
      t2[ORA_NCMAX * ORA_NCMAX];
  FN(m_eq_r_times_m)(x, nc, (R)(1 / ds), a);
  FN(m_eq_d)(e, nc, (R)0.5);
  FN(m_peq_r_times_m)(e, nc, (R)(-0.5), x);
  for (int k = 0; k < nc * nc; k++) { x[k].re += e[k].re; x[k].im += e[k].im; }
  double enorm;
  int nit = 0;
  do {
    nit++;
    FN(m_eq_m_inverse_m)(t1, nc, x, e);
    FN(m_eq_m_times_m)(t2, nc, e, t1);
    FN(m_eq_r_times_m)(e, nc, (R)(-0.5), t2);
    for (int k = 0; k < nc * nc; k++) { x[k].re += e[k].re; x[k].im += e[k].im; }
    enorm = FN(fnorm2)(e, nc);
  } while (nit < 20 && enorm > eps);
  FN(m_eq_r_times_m)(r, nc, (R)sqrt(ds), x);
}

/* ------------------------------------------------------------ v-forms */
void FN(ora_mfunc)(R *r, const R *a, long n, int nc, int which)
{
  const FN(mc) *A = (const FN(mc) *)a;
  FN(mc) *O = (FN(mc) *)r;
  const double eps = sizeof(R) == 4 ? (double)FLT_EPSILON : DBL_EPSILON;
  for (long i = 0; i < n; i++) {
    const FN(mc) *ai = A + i * nc * nc;
    switch (which) {
    case ORA_MF_EXP: FN(exp1)(O + i * nc * nc, ai, nc); break;
    case ORA_MF_SQRT: FN(sqrt1)(O + i * nc * nc, ai, nc, eps); break;
    case ORA_MF_INVERSE: FN(inverse1)(O + i * nc * nc, ai, nc); break;
    default: FN(det1)(O + i, ai, nc); break;
    }
  }
}

#undef CMUL
#undef CMMS
#undef CPMS
#undef EL
#undef FN
#undef CAT2
#undef CAT2_
