/*
 * Test infrastructure (the oracle): precision-generic body of the CPU restatement
 * of QLA 1.9.0's level-1 site operators.  Included twice by qla_oracle.c with
 *   R   = float | double        (site arithmetic type)
 *   SFX = f     | d             (name suffix)
 *
 * Every loop restates the code the reference generator emits, with the same
 * operation order, so that compiled without FP contraction (-ffp-contract=off)
 * the results are bit-identical to the reference library's.
 *
 * Record layout (include/qla_types.h:29-33): a site record is an array of
 * complex numbers, colour-major with spin / column inner:
 *   V[ic], H[ic][is<2], D[ic][is<4], M[ic][jc].
 * A "field" argument is a flat array of records; an optional int32 index
 * array idx_X maps site k to record idx_X[k] (this models both the pointer
 * variants `pX`, where b[k] == &src[idx_b[k]], and the per-operand index
 * variants `xX`, doc/qla.tex:476-487), and an optional gang index j maps loop
 * position i to site k = j[i] (the `x` variants, lib/perl/indirection.pl:66-101).
 */

#define CAT2_(a, b) a##_##b
#define CAT2(a, b) CAT2_(a, b)
#define FN(name) CAT2(name, SFX)

typedef struct { R re, im; } FN(cplx);

/* site index helpers */
static inline long FN(site_)(const int *gang, long i) { return gang ? gang[i] : i; }
static inline long FN(rec_)(const int *idx, long k) { return idx ? idx[k] : k; }

/* ------------------------------------------------------------------------ */
/* eqop accumulate of one complex product, literal restatement of the
 * include/qla_complex.h:326-405 macros (QLA_c_{peq,meq}_{c,ca}_times_{c,ca}).
 * acc is x; conj flags select the macro. */
static inline void FN(cmac_)(FN(cplx) *x, int minus, int ca, int cb,
                             R ar, R ai, R br, R bi)
{
  R re, im;
  if (!ca && !cb) {        /* c_peq_c_times_c  qla_complex.h:330-333 */
    re = (ar*br - ai*bi);
    im = (ar*bi + ai*br);
  } else if (ca && !cb) {  /* c_peq_ca_times_c qla_complex.h:386-389 */
    re = ar*br + ai*bi;
    im = ar*bi - ai*br;
  } else if (!ca && cb) {  /* c_peq_c_times_ca qla_complex.h:366-369 */
    re = ar*br + ai*bi;
    im = ai*br - ar*bi;
  } else {                 /* c_peq_ca_times_ca qla_complex.h:347-350 */
    re = ar*br - ai*bi;
    im = -ar*bi - ai*br;
  }
  if (minus) { x->re -= re; x->im -= im; }
  else       { x->re += re; x->im += im; }
}

/* ------------------------------------------------------------------------ */
/* Left multiplication by a colour matrix:  r (eqop) A * B
 *   A = a or a^dagger (adja),  B = b (nc x ncol) or, for matrix b, b^dagger.
 * Emitter: lib/perl/build_qla.pl:1588-1622 (left mult by colormatrix),
 *          lib/perl/expressions_tensor.pl:766 (print_val_eqop_val_op_val_single).
 * Generated form (e.g. QLA_F3_V_vpeq_M_times_V): per output element,
 *   x = (peq|meq) ? r : 0;  for k: x (+|-)= A(i,k) * B(k,s);  r = x.
 * eqop: 0 eq, 1 peq, 2 meq, 3 eqm.
 */
void FN(ora_lmult)(R *r, const R *a, const R *b, long n, int nc, int ncol,
                   int eqop, int adja, int adjb,
                   const int *idx_a, const int *idx_b, const int *gang)
{
  const long msz = (long)nc * nc;          /* complex numbers per matrix */
  const long bsz = (long)nc * ncol;        /* complex numbers per b record */
  int minus = (eqop == 2 || eqop == 3);
  int load = (eqop == 1 || eqop == 2);
  for (long i = 0; i < n; i++) {
    long k = FN(site_)(gang, i);
    const FN(cplx) *A = (const FN(cplx) *)a + FN(rec_)(idx_a, k) * msz;
    const FN(cplx) *B = (const FN(cplx) *)b + FN(rec_)(idx_b, k) * bsz;
    FN(cplx) *O = (FN(cplx) *)r + k * bsz;
    for (int ic = 0; ic < nc; ic++) {
      for (int s = 0; s < ncol; s++) {
        FN(cplx) x;
        if (load) x = O[ic*ncol + s]; else { x.re = 0.; x.im = 0.; }
        for (int kc = 0; kc < nc; kc++) {
          FN(cplx) av = adja ? A[kc*nc + ic] : A[ic*nc + kc];
          FN(cplx) bv = adjb ? B[s*ncol + kc] : B[kc*ncol + s];
          FN(cmac_)(&x, minus, adja, adjb, av.re, av.im, bv.re, bv.im);
        }
        O[ic*ncol + s] = x;
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Two-operand complex ops of the spin projector, literal restatements of
 * qla_complex.h:287-324 (c_{eq,eqm,peq,meq}_c_{plus,minus}_{c,ic}).
 * kind: 0 c+c, 1 c-c, 2 c+ic, 3 c-ic, 4 copy of a (op 'c'). */
static inline void FN(c2op_)(FN(cplx) *c, int eqop, int kind, FN(cplx) a, FN(cplx) b)
{
  R re = 0, im = 0;
  if (kind == 4) {               /* carith1 {eq,eqm,peq,meq}c, qla_complex.h:147-154 */
    switch (eqop) {
    case 0: c->re = a.re; c->im = a.im; return;
    case 3: c->re = -a.re; c->im = -a.im; return;
    case 1: c->re += a.re; c->im += a.im; return;
    default: c->re -= a.re; c->im -= a.im; return;
    }
  }
  if (eqop == 3) {               /* eqm forms are written out separately */
    switch (kind) {
    case 0: c->re = -a.re - b.re; c->im = -a.im - b.im; return;
    case 1: c->re = -a.re + b.re; c->im = -a.im + b.im; return;
    case 2: c->re = -a.re + b.im; c->im = -a.im - b.re; return;
    default: c->re = -a.re - b.im; c->im = -a.im + b.re; return;
    }
  }
  switch (kind) {
  case 0: re = a.re + b.re; im = a.im + b.im; break;
  case 1: re = a.re - b.re; im = a.im - b.im; break;
  case 2: re = a.re - b.im; im = a.im + b.re; break;
  default: re = a.re + b.im; im = a.im - b.re; break;
  }
  if (eqop == 0) { c->re = re; c->im = im; }
  else if (eqop == 1) { c->re += re; c->im += im; }
  else { c->re -= re; c->im -= im; }
}

/* Spin projection table, restating lib/perl/expressions_gamma.pl:244-275
 * (print_val_assign_spproj_dirs) for a HalfFermion destination:
 * per (sign, mu): for h-spin 0 and 1 the op kind and the two D spins. */
static const int FN(spproj_tab_)[2][5][2][3] = {
  /* sign = +1 */
  { { {2, 0, 3}, {2, 1, 2} },      /* mu 0: c+ic (0,3), c+ic (1,2) */
    { {1, 0, 3}, {0, 1, 2} },      /* mu 1: c-c, c+c */
    { {2, 0, 2}, {3, 1, 3} },      /* mu 2: c+ic, c-ic */
    { {0, 0, 2}, {0, 1, 3} },      /* mu 3: c+c, c+c */
    { {4, 0, 0}, {4, 1, 1} } },    /* mu 4: copy 0, 1 */
  /* sign = -1 (any sign != 1, as in the generated `else` branch) */
  { { {3, 0, 3}, {3, 1, 2} },
    { {0, 0, 3}, {1, 1, 2} },
    { {3, 0, 2}, {2, 1, 3} },
    { {1, 0, 2}, {1, 1, 3} },
    { {4, 2, 2}, {4, 3, 3} } } };

/* H (eqop) spproj(D, mu, sign).  Emitter build_qla.pl:1087-1110,
 * make_code_unary.pl:183-241.  mu outside 0..4 leaves r untouched (the
 * generated switch has no default). */
void FN(ora_spproj)(R *r, const R *a, long n, int nc, int mu, int sign, int eqop,
                    const int *idx_a, const int *gang)
{
  if (mu < 0 || mu > 4) return;
  const int (*t)[3] = FN(spproj_tab_)[sign == 1 ? 0 : 1][mu];
  for (long i = 0; i < n; i++) {
    long k = FN(site_)(gang, i);
    const FN(cplx) *A = (const FN(cplx) *)a + FN(rec_)(idx_a, k) * nc * 4;
    FN(cplx) *O = (FN(cplx) *)r + k * nc * 2;
    for (int ic = 0; ic < nc; ic++)
      for (int h = 0; h < 2; h++)
        FN(c2op_)(&O[ic*2 + h], eqop, t[h][0], A[ic*4 + t[h][1]], A[ic*4 + t[h][2]]);
  }
}

/* One-operand ops of the reconstruction: op 0 '0', 1 'c', 2 '-c', 3 'ic', 4 '-ic'
 * mapped through the carith1 table (lib/perl/headers.pl:136-169) onto
 * qla_complex.h:147-172. */
static inline void FN(c1op_)(FN(cplx) *c, int eqop, int op, FN(cplx) a)
{
  if (op == 0) {
    if (eqop == 0 || eqop == 3) { c->re = 0.0; c->im = 0.0; }
    return;
  }
  int neg = (op == 2 || op == 4);
  int ic = (op == 3 || op == 4);
  /* fold the sign of the op into the eqop exactly as carith1 does */
  int e = eqop;
  if (neg) e = (eqop == 0) ? 3 : (eqop == 3) ? 0 : (eqop == 1) ? 2 : 1;
  if (!ic) {
    switch (e) {
    case 0: c->re = a.re; c->im = a.im; break;
    case 3: c->re = -a.re; c->im = -a.im; break;
    case 1: c->re += a.re; c->im += a.im; break;
    default: c->re -= a.re; c->im -= a.im; break;
    }
  } else {
    switch (e) {
    case 0: c->re = -a.im; c->im = a.re; break;
    case 3: c->re = a.im; c->im = -a.re; break;
    case 1: c->re -= a.im; c->im += a.re; break;
    default: c->re += a.im; c->im -= a.re; break;
    }
  }
}

/* Reconstruction table, restating expressions_gamma.pl:309-337
 * (print_val_assign_sprecon_dirs): per (sign, mu), for D spins 0..3 the op
 * and the source h-spin. */
static const int FN(sprecon_tab_)[2][5][4][2] = {
  { { {1,0}, {1,1}, {4,1}, {4,0} },   /* mu 0: c c -ic -ic ; h 0 1 1 0 */
    { {1,0}, {1,1}, {1,1}, {2,0} },   /* mu 1: c c c -c    ; h 0 1 1 0 */
    { {1,0}, {1,1}, {4,0}, {3,1} },   /* mu 2: c c -ic ic  ; h 0 1 0 1 */
    { {1,0}, {1,1}, {1,0}, {1,1} },   /* mu 3: c c c c     ; h 0 1 0 1 */
    { {1,0}, {1,1}, {0,0}, {0,1} } }, /* mu 4: c c 0 0 */
  { { {1,0}, {1,1}, {3,1}, {3,0} },   /* mu 0: c c ic ic */
    { {1,0}, {1,1}, {2,1}, {1,0} },   /* mu 1: c c -c c */
    { {1,0}, {1,1}, {3,0}, {4,1} },   /* mu 2: c c ic -ic */
    { {1,0}, {1,1}, {2,0}, {2,1} },   /* mu 3: c c -c -c */
    { {0,0}, {0,1}, {1,0}, {1,1} } } }; /* mu 4: 0 0 c c */

/* D (eqop) sprecon(H, mu, sign).  Emitter build_qla.pl:1112-1135. */
void FN(ora_sprecon)(R *r, const R *a, long n, int nc, int mu, int sign, int eqop,
                     const int *idx_a, const int *gang)
{
  if (mu < 0 || mu > 4) return;
  const int (*t)[2] = FN(sprecon_tab_)[sign == 1 ? 0 : 1][mu];
  for (long i = 0; i < n; i++) {
    long k = FN(site_)(gang, i);
    const FN(cplx) *A = (const FN(cplx) *)a + FN(rec_)(idx_a, k) * nc * 2;
    FN(cplx) *O = (FN(cplx) *)r + k * nc * 4;
    for (int ic = 0; ic < nc; ic++)
      for (int s = 0; s < 4; s++)
        FN(c1op_)(&O[ic*4 + s], eqop, t[s][0], A[ic*2 + t[s][1]]);
  }
}

/* ------------------------------------------------------------------------ */
/* r (eqop) a * b with a real scalar read once (`at = *a`), restating
 * build_qla.pl:1256-1292 and qla_complex.h:258-265 (c_{eq,eqm,peq,meq}_c_times_r).
 * ncplx = complex numbers per record. */
void FN(ora_rtimes)(R *r, R a, const R *b, long n, int ncplx, int eqop,
                    const int *idx_b, const int *gang)
{
  for (long i = 0; i < n; i++) {
    long k = FN(site_)(gang, i);
    const FN(cplx) *B = (const FN(cplx) *)b + FN(rec_)(idx_b, k) * ncplx;
    FN(cplx) *O = (FN(cplx) *)r + k * ncplx;
    for (int e = 0; e < ncplx; e++) {
      switch (eqop) {
      case 0: O[e].re = a * B[e].re; O[e].im = a * B[e].im; break;
      case 3: O[e].re = -(a * B[e].re); O[e].im = -(a * B[e].im); break;
      case 1: O[e].re += a * B[e].re; O[e].im += a * B[e].im; break;
      default: O[e].re -= a * B[e].re; O[e].im -= a * B[e].im; break;
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Global norm2, reference semantics (build_qla.pl:2089-2155,
 * make_code_unary.pl:318-365): each |z|^2 = re*re + im*im evaluated in the site
 * type R, promoted, and summed sequentially in double (datatypes.pl:355-358). */
double FN(ora_norm2_ref)(const R *a, long n, int ncplx, const int *idx_a, const int *gang)
{
  double sum = 0.;
  for (long i = 0; i < n; i++) {
    long k = FN(site_)(gang, i);
    const FN(cplx) *A = (const FN(cplx) *)a + FN(rec_)(idx_a, k) * ncplx;
    for (int e = 0; e < ncplx; e++) {
      FN(cplx) at = A[e];
      sum += at.re*at.re + at.im*at.im;
    }
  }
  return sum;
}

/* Global inner product sum conj(a).b, reference semantics
 * (build_qla.pl:2196-2360, make_code_binary.pl:110-172): the operands are
 * promoted to double before the product (QLA_DF_c), qla_complex.h:386-389. */
void FN(ora_dot_ref)(double *out2, const R *a, const R *b, long n, int ncplx,
                     const int *idx_a, const int *idx_b, const int *gang)
{
  double sre = 0., sim = 0.;
  for (long i = 0; i < n; i++) {
    long k = FN(site_)(gang, i);
    const FN(cplx) *A = (const FN(cplx) *)a + FN(rec_)(idx_a, k) * ncplx;
    const FN(cplx) *B = (const FN(cplx) *)b + FN(rec_)(idx_b, k) * ncplx;
    for (int e = 0; e < ncplx; e++) {
      double ar = A[e].re, ai = A[e].im, br = B[e].re, bi = B[e].im;
      sre += ar*br + ai*bi;
      sim += ar*bi - ai*br;
    }
  }
  out2[0] = sre; out2[1] = sim;
}

/* Per-site complex dot field  C[k] = sum_e conj(a_e) b_e  (QLA_F3_C_veq_D_dot_D):
 * double temporary per site (QLA_D_Complex x), rounded to the field type. */
void FN(ora_dot_field)(R *r, const R *a, const R *b, long n, int ncplx,
                       const int *idx_a, const int *idx_b, const int *gang)
{
  for (long i = 0; i < n; i++) {
    long k = FN(site_)(gang, i);
    const FN(cplx) *A = (const FN(cplx) *)a + FN(rec_)(idx_a, k) * ncplx;
    const FN(cplx) *B = (const FN(cplx) *)b + FN(rec_)(idx_b, k) * ncplx;
    double xre = 0., xim = 0.;
    for (int e = 0; e < ncplx; e++) {
      double ar = A[e].re, ai = A[e].im, br = B[e].re, bi = B[e].im;
      xre += ar*br + ai*bi;
      xim += ar*bi - ai*br;
    }
    r[2*k] = (R)xre; r[2*k + 1] = (R)xim;
  }
}

/* ------------------------------------------------------------------------ */
/* DiracPropagator products and spin trace (build_qla.pl:1588-1661, 942-968):
 * kind 0: r (eqop) A P',  1: r (eqop) P' A,  2: r (eqop) P' P'',  3: M (eqop) spintrace(P)
 * with A = M or M^+ (ca / cb), P' = P or P^+ (P^+[i][s][j][t] = conj P[j][t][i][s]);
 * per output element x = (peq|meq ? r : 0), then x (+|-)= a*b over k (kc, then ks). */
static inline long FN(pix_)(int i, int s, int j, int t, int adj, int nc)
{
  return adj ? ((j * 4 + t) * nc + i) * 4 + s : ((i * 4 + s) * nc + j) * 4 + t;
}
static inline long FN(mix_)(int i, int j, int adj, int nc) { return adj ? j * nc + i : i * nc + j; }

void FN(ora_prop_n)(int nc, int kind, int ca, int cb, int eqop, R *r, const R *a, const R *b, long n,
                    const int *idx_a, const int *idx_b, const int *gang)
{
  const int minus = (eqop == 2 || eqop == 3), load = (eqop == 1 || eqop == 2);
  const long nm = nc * nc, np_ = 16 * nc * nc;
  const long ra = (kind == 0) ? nm : np_, rb = (kind == 1) ? nm : np_;
  const int nel = (kind == 3) ? nm : np_;
  for (long i = 0; i < n; i++) {
    long k = FN(site_)(gang, i);
    const FN(cplx) *A = (const FN(cplx) *)a + FN(rec_)(idx_a, k) * ra;
    const FN(cplx) *B = (kind == 3) ? 0 : (const FN(cplx) *)b + FN(rec_)(idx_b, k) * rb;
    FN(cplx) *O = (FN(cplx) *)r + k * nel;
    for (int e = 0; e < nel; e++) {
      FN(cplx) x;
      if (load) x = O[e]; else { x.re = 0.; x.im = 0.; }
      if (kind == 3) {
        int ic = e / nc, jc = e % nc;
        for (int s2 = 0; s2 < 4; s2++) {
          FN(cplx) v = A[FN(pix_)(ic, s2, jc, s2, 0, nc)];
          if (minus) { x.re -= v.re; x.im -= v.im; } else { x.re += v.re; x.im += v.im; }
        }
      } else {
        int ic = e / (16 * nc), is = (e / (4 * nc)) % 4, jc = (e / 4) % nc, js = e % 4;
        for (int kc = 0; kc < nc; kc++) {
          if (kind == 2) {
            for (int ks = 0; ks < 4; ks++) {
              FN(cplx) u = A[FN(pix_)(ic, is, kc, ks, ca, nc)], v = B[FN(pix_)(kc, ks, jc, js, cb, nc)];
              FN(cmac_)(&x, minus, ca, cb, u.re, u.im, v.re, v.im);
            }
          } else if (kind == 0) {
            FN(cplx) u = A[FN(mix_)(ic, kc, ca, nc)], v = B[FN(pix_)(kc, is, jc, js, cb, nc)];
            FN(cmac_)(&x, minus, ca, cb, u.re, u.im, v.re, v.im);
          } else {
            FN(cplx) u = A[FN(pix_)(ic, is, kc, js, ca, nc)], v = B[FN(mix_)(kc, jc, cb, nc)];
            FN(cmac_)(&x, minus, ca, cb, u.re, u.im, v.re, v.im);
          }
        }
      }
      O[e] = x;
    }
  }
}

void FN(ora_prop)(int kind, int ca, int cb, int eqop, R *r, const R *a, const R *b, long n,
                  const int *idx_a, const int *idx_b, const int *gang)
{
  FN(ora_prop_n)(3, kind, ca, cb, eqop, r, a, b, n, idx_a, idx_b, gang);
}

#undef FN
#undef CAT2
#undef CAT2_
