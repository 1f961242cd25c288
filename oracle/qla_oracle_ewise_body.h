/*
 * Test infrastructure (the oracle) -- NOT product code.
 * Element-wise level-1 families restated from the QLA complex macros
 * (include/qla_complex.h:140-460) as the generated loops use them
 * (lib/perl/build_qla.pl:403-469, 1256-1420, 2358-2460): every output
 * complex number is one macro applied to same-position source elements, in
 * the site precision R, with no FMA contraction.  Included twice by
 * qla_oracle_ewise.c (R = float / double).
 */
#define CAT2_(a, b) a##_##b
#define CAT2(a, b) CAT2_(a, b)
#define FN(name) CAT2(name, SFX)

typedef struct { R re, im; } FN(ec);

/* element e of the transposed record: perm 1 the nc x nc colour matrix,
 * perm 2 the (colour, spin) x (colour, spin) propagator of blocks 4 nc */
static int FN(eperm)(int perm, int e, int nc)
{
  if (perm == 1) return (e % nc) * nc + e / nc;
  if (perm == 2) return (e % (4 * nc)) * (4 * nc) + e / (4 * nc);
  return e;
}

/* shape codes as the product's EwShape; eqop 0 eq, 1 peq, 2 meq, 3 eqm */
static FN(ec) FN(eapply)(int shape, int eqop, FN(ec) x, FN(ec) s, FN(ec) b, FN(ec) c)
{
  FN(ec) r;
  switch (shape) {
  case 0:  /* QLA_c_(eqop)_c */
    if (eqop == 0) r = b;
    else if (eqop == 3) { r.re = -b.re; r.im = -b.im; }
    else if (eqop == 1) { r.re = x.re + b.re; r.im = x.im + b.im; }
    else { r.re = x.re - b.re; r.im = x.im - b.im; }
    return r;
  case 1:  /* QLA_c_(eqop)_ca */
    if (eqop == 0) { r.re = b.re; r.im = -b.im; }
    else if (eqop == 3) { r.re = -b.re; r.im = b.im; }
    else if (eqop == 1) { r.re = x.re + b.re; r.im = x.im - b.im; }
    else { r.re = x.re - b.re; r.im = x.im + b.im; }
    return r;
  case 2:  /* QLA_c_(eqop)_ic */
    if (eqop == 0) { r.re = -b.im; r.im = b.re; }
    else if (eqop == 3) { r.re = b.im; r.im = -b.re; }
    else if (eqop == 1) { r.re = x.re - b.im; r.im = x.im + b.re; }
    else { r.re = x.re + b.im; r.im = x.im - b.re; }
    return r;
  case 3:  /* QLA_c_(eqop)_c_times_c(r, s, b) */
    if (eqop == 0) { r.re = s.re*b.re - s.im*b.im; r.im = s.re*b.im + s.im*b.re; }
    else if (eqop == 3) { r.re = -s.re*b.re + s.im*b.im; r.im = -s.re*b.im - s.im*b.re; }
    else if (eqop == 1) { r.re = x.re + (s.re*b.re - s.im*b.im); r.im = x.im + (s.re*b.im + s.im*b.re); }
    else { r.re = x.re - (s.re*b.re - s.im*b.im); r.im = x.im - (s.re*b.im + s.im*b.re); }
    return r;
  case 4:  /* QLA_c_(eqop)_c_times_ca(r, s, b) */
    if (eqop == 0) { r.re = s.re*b.re + s.im*b.im; r.im = s.im*b.re - s.re*b.im; }
    else if (eqop == 3) { r.re = -s.re*b.re - s.im*b.im; r.im = -s.im*b.re + s.re*b.im; }
    else if (eqop == 1) { r.re = x.re + (s.re*b.re + s.im*b.im); r.im = x.im + (s.im*b.re - s.re*b.im); }
    else { r.re = x.re - (s.re*b.re + s.im*b.im); r.im = x.im - (s.im*b.re - s.re*b.im); }
    return r;
  case 5:  /* QLA_c_(eqop)_ca_times_c(r, s, b) */
    if (eqop == 0) { r.re = s.re*b.re + s.im*b.im; r.im = s.re*b.im - s.im*b.re; }
    else if (eqop == 3) { r.re = -s.re*b.re - s.im*b.im; r.im = -s.re*b.im + s.im*b.re; }
    else if (eqop == 1) { r.re = x.re + (s.re*b.re + s.im*b.im); r.im = x.im + (s.re*b.im - s.im*b.re); }
    else { r.re = x.re - (s.re*b.re + s.im*b.im); r.im = x.im - (s.re*b.im - s.im*b.re); }
    return r;
  case 6:  /* QLA_c_(eqop)_ca_times_ca(r, s, b) */
    if (eqop == 0) { r.re = s.re*b.re - s.im*b.im; r.im = -s.re*b.im - s.im*b.re; }
    else if (eqop == 3) { r.re = -s.re*b.re + s.im*b.im; r.im = s.re*b.im + s.im*b.re; }
    else if (eqop == 1) { r.re = x.re + (s.re*b.re - s.im*b.im); r.im = x.im + (-s.re*b.im - s.im*b.re); }
    else { r.re = x.re - (s.re*b.re - s.im*b.im); r.im = x.im - (-s.re*b.im - s.im*b.re); }
    return r;
  case 7:  /* QLA_c_(eqop)_r_times_c(r, s, b) */
    if (eqop == 0) { r.re = s.re*b.re; r.im = s.re*b.im; }
    else if (eqop == 3) { r.re = -(s.re*b.re); r.im = -(s.re*b.im); }
    else if (eqop == 1) { r.re = x.re + s.re*b.re; r.im = x.im + s.re*b.im; }
    else { r.re = x.re - s.re*b.re; r.im = x.im - s.re*b.im; }
    return r;
  case 8:  /* QLA_c_(eqop)_r_times_ca(r, s, b) */
    if (eqop == 0) { r.re = s.re*b.re; r.im = -(s.re*b.im); }
    else if (eqop == 3) { r.re = -(s.re*b.re); r.im = s.re*b.im; }
    else if (eqop == 1) { r.re = x.re + s.re*b.re; r.im = x.im - s.re*b.im; }
    else { r.re = x.re - s.re*b.re; r.im = x.im + s.re*b.im; }
    return r;
  case 9: r.re = b.re + c.re; r.im = b.im + c.im; return r;          /* c_eq_c_plus_c */
  case 10: r.re = b.re - c.re; r.im = b.im - c.im; return r;         /* c_eq_c_minus_c */
  case 11: r.re = s.re*b.re + c.re; r.im = s.re*b.im + c.im; return r; /* c_eq_r_times_c_plus_c */
  case 12: r.re = s.re*b.re - c.re; r.im = s.re*b.im - c.im; return r; /* c_eq_r_times_c_minus_c */
  case 13:                                                           /* c_eq_c_times_c_plus_c */
    r.re = s.re*b.re - s.im*b.im + c.re; r.im = s.re*b.im + s.im*b.re + c.im; return r;
  default:                                                           /* c_eq_c_times_c_minus_c */
    r.re = s.re*b.re - s.im*b.im - c.re; r.im = s.re*b.im + s.im*b.re - c.im; return r;
  }
}

/* r[k] (eqop)= shape(s, b[k] in perm order, c[k]) over the records k = gang[i]
 * (or i); b, c, s each either contiguous or gathered through idx_* (the
 * pointer form); scal_kind 0 none, 1 constant (sre, sim), 2 per-site complex
 * field s, 3 per-site real field s */
void FN(ora_ewise_n)(int nc, int shape, int perm, int eqop, R *r, const R *b, const R *c, const R *s,
                     int scal_kind, R sre, R sim, long n, int ne, const int *idx_b, const int *idx_c,
                     const int *idx_s, const int *gang)
{
  const FN(ec) *B = (const FN(ec) *)b, *C = (const FN(ec) *)c;
  FN(ec) *O = (FN(ec) *)r;
  for (long i = 0; i < n; i++) {
    const long k = gang ? gang[i] : i;
    const long kb = idx_b ? idx_b[k] : k, kc = idx_c ? idx_c[k] : k, ks = idx_s ? idx_s[k] : k;
    FN(ec) sv; sv.re = 0; sv.im = 0;
    if (scal_kind == 1) { sv.re = sre; sv.im = sim; }
    else if (scal_kind == 2) { sv = ((const FN(ec) *)s)[ks]; }
    else if (scal_kind == 3) { sv.re = s[ks]; }
    for (int e = 0; e < ne; e++) {
      FN(ec) bv = B[kb * ne + FN(eperm)(perm, e, nc)], cv; cv.re = 0; cv.im = 0;
      if (C) cv = C[kc * ne + e];
      O[k * ne + e] = FN(eapply)(shape, eqop, O[k * ne + e], sv, bv, cv);
    }
  }
}

void FN(ora_ewise)(int shape, int perm, int eqop, R *r, const R *b, const R *c, const R *s, int scal_kind,
                   R sre, R sim, long n, int ne, const int *idx_b, const int *idx_c, const int *idx_s,
                   const int *gang)
{
  FN(ora_ewise_n)(3, shape, perm, eqop, r, b, c, s, scal_kind, sre, sim, n, ne, idx_b, idx_c, idx_s, gang);
}

/* M (eqop)= a b^+ per site (QLA_c_(eqop)_c_times_ca(r_ij, a_i, b_j)) */
void FN(ora_outer_n)(int nc, int eqop, R *r, const R *a, const R *b, long n, const int *idx_a, const int *idx_b,
                     const int *gang)
{
  const FN(ec) *A = (const FN(ec) *)a, *B = (const FN(ec) *)b;
  FN(ec) *O = (FN(ec) *)r;
  FN(ec) z; z.re = 0; z.im = 0;
  const int m = nc * nc;
  for (long i = 0; i < n; i++) {
    const long k = gang ? gang[i] : i;
    const long ka = idx_a ? idx_a[k] : k, kb = idx_b ? idx_b[k] : k;
    for (int e = 0; e < m; e++)
      O[k * m + e] = FN(eapply)(4, eqop, O[k * m + e], A[ka * nc + e / nc], B[kb * nc + e % nc], z);
  }
}

void FN(ora_outer)(int eqop, R *r, const R *a, const R *b, long n, const int *idx_a, const int *idx_b,
                   const int *gang)
{
  FN(ora_outer_n)(3, eqop, r, a, b, n, idx_a, idx_b, gang);
}

/* site-local dot products (kind as the product's LdKind), accumulated in
 * double from promoted elements (QLA_DF_c), then QLA_FD_c and the eqop; real
 * outputs (kind >= 3) combine r and x in double */
void FN(ora_ldot_n)(int nc, int kind, int perm, int eqop, R *r, const R *a, const R *b, long n, int ne,
                    const int *idx_a, const int *idx_b, const int *gang)
{
  const FN(ec) *A = (const FN(ec) *)a, *B = (const FN(ec) *)(b ? b : a);
  for (long i = 0; i < n; i++) {
    const long k = gang ? gang[i] : i;
    const long ka = idx_a ? idx_a[k] : k, kb = (kind == 4) ? ka : (idx_b ? idx_b[k] : k);
    double xr = 0., xi = 0.;
    for (int e = 0; e < ne; e++) {
      double ur, ui, vr, vi;
      int ea = e, eb = e;
      if (kind == 2) ea = FN(eperm)(perm, e, nc);
      if (kind == 1) eb = FN(eperm)(perm, e, nc);
      ur = A[ka * ne + ea].re; ui = A[ka * ne + ea].im;
      vr = B[kb * ne + eb].re; vi = B[kb * ne + eb].im;
      if (kind == 0 || kind == 3 || kind == 4) {       /* peq_ca_times_c */
        xr += ur*vr + ui*vi;
        xi += ur*vi - ui*vr;
      } else if (kind == 1) {                          /* peq_ca_times_ca */
        xr += ur*vr - ui*vi;
        xi += -ur*vi - ui*vr;
      } else {                                         /* peq_c_times_c */
        xr += (ur*vr - ui*vi);
        xi += (ur*vi + ui*vr);
      }
    }
    if (kind >= 3) {
      if (eqop == 0) r[k] = xr;
      else if (eqop == 3) r[k] = -xr;
      else if (eqop == 1) r[k] += xr;
      else r[k] -= xr;
    } else {
      FN(ec) *q = (FN(ec) *)r + k, t;
      t.re = (R)xr; t.im = (R)xi;
      if (eqop == 0) *q = t;
      else if (eqop == 3) { q->re = -t.re; q->im = -t.im; }
      else if (eqop == 1) { q->re += t.re; q->im += t.im; }
      else { q->re -= t.re; q->im -= t.im; }
    }
  }
}

void FN(ora_ldot)(int kind, int perm, int eqop, R *r, const R *a, const R *b, long n, int ne, const int *idx_a,
                  const int *idx_b, const int *gang)
{
  FN(ora_ldot_n)(3, kind, perm, eqop, r, a, b, n, ne, idx_a, idx_b, gang);
}

#undef FN
#undef CAT2
#undef CAT2_
