/*
 * Test infrastructure (the oracle) -- NOT product code.
 * Site-field families restated from the loops the reference generator emits:
 * constant / diagonal / zero fills (lib/perl/build_qla.pl:2561-2618),
 * copymask (:2058-2084), array components, colour columns and Dirac vectors
 * (:767-931), gamma multiplication (:1358-1412 with the basis and row /
 * column selection of lib/perl/expressions_gamma.pl:59-170, 384-470), trace
 * and antihermitian part (:933-1064), global reductions of DiracPropagators
 * and of the adjoint-form products (:2089-2272) and global sums
 * (:2449-2521), in the reference's element and site order.  Included twice
 * by qla_oracle_sitefield.c (R = float / double).
 */
#define CAT2_(a, b) a##_##b
#define CAT2(a, b) CAT2_(a, b)
#define FN(name) CAT2(name, SFX)

typedef struct { R re, im; } FN(sc);

/* component of (ic, is, jc, js) in a record of letter t with nc colours
 * (include/qla_types.h:38-42) */
static int FN(selem)(char t, int ic, int is, int jc, int js, int nc)
{
  switch (t) {
  case 'V': return ic;
  case 'H': return ic * 2 + is;
  case 'D': return ic * 4 + is;
  case 'M': return ic * nc + jc;
  case 'P': return ((ic * 4 + is) * nc + jc) * 4 + js;
  default: return 0;
  }
}

static int FN(sne)(int t, int nc)
{
  switch (t) {
  case 'V': return nc;
  case 'H': return 2 * nc;
  case 'D': return 4 * nc;
  case 'M': return nc * nc;
  case 'P': return 16 * nc * nc;
  default: return 1;
  }
}

/* r[k] (eqop)= a (one record): QLA_c_(eqop)_c per component */
void FN(ora_fill)(int eqop, R *r, const R *a, long n, int ne, const int *gang)
{
  FN(sc) *Rr = (FN(sc) *)r;
  const FN(sc) *A = (const FN(sc) *)a;
  for (long i = 0; i < n; i++) {
    const long k = gang ? gang[i] : i;
    for (int e = 0; e < ne; e++) {
      FN(sc) *q = &Rr[k * ne + e];
      if (eqop == 0) *q = A[e];
      else if (eqop == 3) { q->re = -A[e].re; q->im = -A[e].im; }
      else if (eqop == 1) { q->re += A[e].re; q->im += A[e].im; }
      else { q->re -= A[e].re; q->im -= A[e].im; }
    }
  }
}

/* M r[k] (eqop)= c * 1: QLA_c_(eqop)_r(r_ij, 0.) for all i, j, then
 * QLA_c_(eqop)_c(r_ii, c) (include/qla_complex.h:140-156) */
void FN(ora_diagfill_n)(int nc, int eqop, R *r, const R *c, long n, const int *gang)
{
  FN(sc) *Rr = (FN(sc) *)r;
  const FN(sc) at = *(const FN(sc) *)c;
  const int m = nc * nc;
  for (long i = 0; i < n; i++) {
    const long k = gang ? gang[i] : i;
    for (int ic = 0; ic < nc; ic++) {
      for (int jc = 0; jc < nc; jc++) {
        FN(sc) *q = &Rr[k * m + ic * nc + jc];
        if (eqop == 0) { q->re = 0.; q->im = 0.; }
        else if (eqop == 3) { q->re = -(0.); q->im = 0.; }
        else if (eqop == 1) q->re += 0.;
        else q->re -= 0.;
      }
      FN(sc) *d = &Rr[k * m + ic * (nc + 1)];
      if (eqop == 0) *d = at;
      else if (eqop == 3) { d->re = -at.re; d->im = -at.im; }
      else if (eqop == 1) { d->re += at.re; d->im += at.im; }
      else { d->re -= at.re; d->im -= at.im; }
    }
  }
}

void FN(ora_diagfill)(int eqop, R *r, const R *c, long n, const int *gang)
{
  FN(ora_diagfill_n)(3, eqop, r, c, n, gang);
}

void FN(ora_zero)(R *r, long n, int ne, const int *gang)
{
  FN(sc) *Rr = (FN(sc) *)r;
  for (long i = 0; i < n; i++) {
    const long k = gang ? gang[i] : i;
    for (int e = 0; e < ne; e++) { Rr[k * ne + e].re = 0.; Rr[k * ne + e].im = 0.; }
  }
}

/* if (b[k]) r[k] = a[k] (pointer forms gathered through idx_a / idx_m) */
void FN(ora_mask)(R *r, const R *a, const int *m, long n, int ne, const int *idx_a, const int *idx_m,
                  const int *gang)
{
  FN(sc) *Rr = (FN(sc) *)r;
  const FN(sc) *A = (const FN(sc) *)a;
  for (long i = 0; i < n; i++) {
    const long k = gang ? gang[i] : i;
    const long ka = idx_a ? idx_a[k] : k, km = idx_m ? idx_m[k] : k;
    if (m[km])
      for (int e = 0; e < ne; e++) Rr[k * ne + e] = A[ka * ne + e];
  }
}

/* what: 'e' array component, 'c' colour column, 'd' Dirac vector; dst / src
 * are the record letters ('C' a single complex number) */
void FN(ora_component_n)(int nc, int what, int dst, int src, R *r, const R *a, int i_c, int i_s, int j_c,
                         int j_s, long n, const int *idx_a, const int *gang)
{
  const int nr = FN(sne)(dst, nc), na = FN(sne)(src, nc);
  FN(sc) *Rr = (FN(sc) *)r;
  const FN(sc) *A = (const FN(sc) *)a;
  for (long i = 0; i < n; i++) {
    const long k = gang ? gang[i] : i;
    const long ka = idx_a ? idx_a[k] : k;
    FN(sc) *rr = &Rr[k * nr];
    const FN(sc) *aa = &A[ka * na];
    if (what == 'e') {
      if (dst == 'C') rr[0] = aa[FN(selem)((char)src, i_c, i_s, j_c, j_s, nc)];
      else rr[FN(selem)((char)dst, i_c, i_s, j_c, j_s, nc)] = aa[0];
    } else if (what == 'c') {
      for (int ic = 0; ic < nc; ic++) {
        if (dst == 'V') rr[ic] = aa[FN(selem)((char)src, ic, i_s, j_c, j_s, nc)];
        else rr[FN(selem)((char)dst, ic, i_s, j_c, j_s, nc)] = aa[ic];
      }
    } else {
      for (int ic = 0; ic < nc; ic++)
        for (int is = 0; is < 4; is++) {
          if (dst == 'D') rr[FN(selem)('D', ic, is, 0, 0, nc)] = aa[FN(selem)('P', ic, is, j_c, j_s, nc)];
          else rr[FN(selem)('P', ic, is, j_c, j_s, nc)] = aa[FN(selem)('D', ic, is, 0, 0, nc)];
        }
    }
  }
}

void FN(ora_component)(int what, int dst, int src, R *r, const R *a, int i_c, int i_s, int j_c, int j_s, long n,
                       const int *idx_a, const int *gang)
{
  FN(ora_component_n)(3, what, dst, src, r, a, i_c, i_s, j_c, j_s, n, idx_a, gang);
}

/* gamma_mu as a product of the basis matrices for the set bits of mu
 * (expressions_gamma.pl:67-134); entries (re, im) */
static void FN(gamma_of)(int mu, int g[4][4][2])
{
  static const int B[4][4][4][2] = {
    {{{0,0},{0,0},{0,0},{0,1}}, {{0,0},{0,0},{0,1},{0,0}}, {{0,0},{0,-1},{0,0},{0,0}}, {{0,-1},{0,0},{0,0},{0,0}}},
    {{{0,0},{0,0},{0,0},{-1,0}}, {{0,0},{0,0},{1,0},{0,0}}, {{0,0},{1,0},{0,0},{0,0}}, {{-1,0},{0,0},{0,0},{0,0}}},
    {{{0,0},{0,0},{0,1},{0,0}}, {{0,0},{0,0},{0,0},{0,-1}}, {{0,-1},{0,0},{0,0},{0,0}}, {{0,0},{0,1},{0,0},{0,0}}},
    {{{0,0},{0,0},{1,0},{0,0}}, {{0,0},{0,0},{0,0},{1,0}}, {{1,0},{0,0},{0,0},{0,0}}, {{0,0},{1,0},{0,0},{0,0}}}};
  int r[4][4][2] = {{{0}}};
  for (int d = 0; d < 4; d++) r[d][d][0] = 1;
  for (int b = 0; b < 4; b++) {
    if (!(mu & (1 << b))) continue;
    int t[4][4][2] = {{{0}}};
    for (int x = 0; x < 4; x++)
      for (int y = 0; y < 4; y++)
        for (int z = 0; z < 4; z++) {
          t[x][y][0] += r[x][z][0] * B[b][z][y][0] - r[x][z][1] * B[b][z][y][1];
          t[x][y][1] += r[x][z][0] * B[b][z][y][1] + r[x][z][1] * B[b][z][y][0];
        }
    for (int x = 0; x < 4; x++)
      for (int y = 0; y < 4; y++) { r[x][y][0] = t[x][y][0]; r[x][y][1] = t[x][y][1]; }
  }
  for (int x = 0; x < 4; x++)
    for (int y = 0; y < 4; y++) { g[x][y][0] = r[x][y][0]; g[x][y][1] = r[x][y][1]; }
}

/* QLA_c_eq_c / eqm_c / eq_ic / eqm_ic by the entry (1, -1, i, -i) */
static FN(sc) FN(gmul)(const int *ent, FN(sc) a)
{
  FN(sc) r;
  if (ent[0] == 1) r = a;
  else if (ent[0] == -1) { r.re = -a.re; r.im = -a.im; }
  else if (ent[1] == 1) { r.re = -a.im; r.im = a.re; }
  else { r.re = a.im; r.im = -a.re; }
  return r;
}

/* left (right == 0): r(.., s, ..) = G[s][t] a(.., t, ..) on the first spin
 * index of a D (ne 12) or P (ne 144); right: r(.., s) = a(.., t) G[t][s] on
 * the last spin index of a P.  mu outside 0..15 leaves r unchanged. */
void FN(ora_gamma_n)(int nc, int right, int ne, int mu, R *r, const R *a, long n, const int *idx_a,
                     const int *gang)
{
  if (mu < 0 || mu > 15) return;
  int g[4][4][2];
  FN(gamma_of)(mu, g);
  int src[4], ent[4][2];
  for (int s = 0; s < 4; s++)
    for (int t = 0; t < 4; t++) {
      const int *v = right ? g[t][s] : g[s][t];
      if (v[0] || v[1]) { src[s] = t; ent[s][0] = v[0]; ent[s][1] = v[1]; }
    }
  FN(sc) *Rr = (FN(sc) *)r;
  const FN(sc) *A = (const FN(sc) *)a;
  for (long i = 0; i < n; i++) {
    const long k = gang ? gang[i] : i;
    const long ka = idx_a ? idx_a[k] : k;
    for (int ic = 0; ic < nc; ic++) {
      if (ne == 4 * nc) {
        for (int s = 0; s < 4; s++)
          Rr[k * ne + FN(selem)('D', ic, s, 0, 0, nc)] = FN(gmul)(ent[s], A[ka * ne + FN(selem)('D', ic, src[s], 0, 0, nc)]);
      } else {
        for (int is = 0; is < 4; is++)
          for (int jc = 0; jc < nc; jc++)
            for (int js = 0; js < 4; js++) {
              const int de = FN(selem)('P', ic, is, jc, js, nc);
              const int se = right ? FN(selem)('P', ic, is, jc, src[js], nc) : FN(selem)('P', ic, src[is], jc, js, nc);
              const int *en = right ? ent[js] : ent[is];
              Rr[k * ne + de] = FN(gmul)(en, A[ka * ne + se]);
            }
      }
    }
  }
}

void FN(ora_gamma)(int right, int ne, int mu, R *r, const R *a, long n, const int *idx_a, const int *gang)
{
  FN(ora_gamma_n)(3, right, ne, mu, r, a, n, idx_a, gang);
}

/* kind 0: C trace, 1: Re trace, 2: Im trace, 3: traceless antihermitian part */
void FN(ora_trace_n)(int nc, int kind, R *r, const R *a, long n, const int *idx_a, const int *gang)
{
  const FN(sc) *A = (const FN(sc) *)a;
  for (long i = 0; i < n; i++) {
    const long k = gang ? gang[i] : i;
    const long ka = idx_a ? idx_a[k] : k;
    const int mm = nc * nc;
    const FN(sc) *m = &A[ka * mm];
    if (kind == 0) {
      FN(sc) x;
      x.re = 0.; x.im = 0.;
      for (int c = 0; c < nc; c++) { x.re += m[c * (nc + 1)].re; x.im += m[c * (nc + 1)].im; }
      ((FN(sc) *)r)[k] = x;
    } else if (kind == 1 || kind == 2) {
      R x = 0.;
      for (int c = 0; c < nc; c++) x += (kind == 1) ? m[c * (nc + 1)].re : m[c * (nc + 1)].im;
      r[k] = x;
    } else {
      FN(sc) *o = (FN(sc) *)r + k * mm;
      R x = 0.;
      for (int c = 0; c < nc; c++) x += m[c * (nc + 1)].im;
      x = x / nc;
      for (int c = 0; c < nc; c++) {
        R x2 = m[c * (nc + 1)].im;
        x2 = x2 - x;
        o[c * (nc + 1)].re = 0.;
        o[c * (nc + 1)].im = x2;
      }
      for (int ic = 0; ic < nc - 1; ic++)
        for (int jc = ic + 1; jc < nc; jc++) {
          FN(sc) x1, x2;
          x1.re = m[ic * nc + jc].re - m[jc * nc + ic].re;
          x1.im = m[ic * nc + jc].im + m[jc * nc + ic].im;
          x2.re = x1.re * 0.5;
          x2.im = x1.im * 0.5;
          o[ic * nc + jc] = x2;
          o[jc * nc + ic].re = -x2.re;
          o[jc * nc + ic].im = x2.im;
        }
    }
  }
}

void FN(ora_trace)(int kind, R *r, const R *a, long n, const int *idx_a, const int *gang)
{
  FN(ora_trace_n)(3, kind, r, a, n, idx_a, gang);
}

/* global reductions in the reference's order: one double sum over all sites
 * and components.  kind as the product's LdKind: 0 X_dot_X (terms conj(a) b
 * promoted), 2 Xa_dot_X (a in perm order times b, no conjugation), 3 re of
 * X_dot_X, 4 norm2 (QLA_norm2_c of the site-precision element, evaluated in
 * R, then added in double).  out2 = (re, im) in double before the final
 * rounding. */
void FN(ora_gdot_n)(int nc, int kind, int perm, double *out2, const R *a, const R *b, long n, int ne,
                    const int *idx_a, const int *idx_b, const int *gang)
{
  const FN(sc) *A = (const FN(sc) *)a, *Bv = (const FN(sc) *)(b ? b : a);
  double sr = 0., si = 0.;
  for (long i = 0; i < n; i++) {
    const long k = gang ? gang[i] : i;
    const long ka = idx_a ? idx_a[k] : k, kb = idx_b ? idx_b[k] : k;
    for (int e = 0; e < ne; e++) {
      if (kind == 4) {
        const FN(sc) at = A[ka * ne + e];
        sr += at.re * at.re + at.im * at.im;
        continue;
      }
      const int bl = (perm == 1) ? nc : 4 * nc;
      const int ea = (kind == 2) ? (e % bl) * bl + e / bl : e;
      const double ur = A[ka * ne + ea].re, ui = A[ka * ne + ea].im;
      const double vr = Bv[kb * ne + e].re, vi = Bv[kb * ne + e].im;
      if (kind == 2) {
        sr += ur * vr - ui * vi;
        si += ur * vi + ui * vr;
      } else {
        sr += ur * vr + ui * vi;
        if (kind == 0) si += ur * vi - ui * vr;
      }
    }
  }
  out2[0] = sr;
  out2[1] = si;
}

void FN(ora_gdot)(int kind, int perm, double *out2, const R *a, const R *b, long n, int ne, const int *idx_a,
                  const int *idx_b, const int *gang)
{
  FN(ora_gdot_n)(3, kind, perm, out2, a, b, n, ne, idx_a, idx_b, gang);
}

/* out = sum over the sites of a, each component in double (the caller
 * rounds it to the output precision: R for F3 / D3, double for DF3) */
void FN(ora_gsum)(double *out, const R *a, long n, int ne, const int *idx_a, const int *gang)
{
  for (int c = 0; c < 2 * ne; c++) out[c] = 0.;
  for (long i = 0; i < n; i++) {
    const long k = gang ? gang[i] : i;
    const long ka = idx_a ? idx_a[k] : k;
    for (int c = 0; c < 2 * ne; c++) out[c] += (double)a[ka * 2 * ne + c];
  }
}

#undef FN
#undef CAT2
#undef CAT2_
