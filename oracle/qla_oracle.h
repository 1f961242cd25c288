/*
 * Test infrastructure (the oracle) -- NOT product code.
 * Declarations of the CPU restatement in qla_oracle.c / qla_oracle_body.h.
 * eqop codes: 0 eq, 1 peq, 2 meq, 3 eqm.  Index arrays may be NULL.
 */
#ifndef QLA_ORACLE_H
#define QLA_ORACLE_H

#define ORA_DECL(SFX, R)                                                           \
void ora_lmult_##SFX(R *r, const R *a, const R *b, long n, int nc, int ncol,      \
                     int eqop, int adja, int adjb,                                \
                     const int *idx_a, const int *idx_b, const int *gang);        \
void ora_spproj_##SFX(R *r, const R *a, long n, int nc, int mu, int sign,        \
                      int eqop, const int *idx_a, const int *gang);               \
void ora_sprecon_##SFX(R *r, const R *a, long n, int nc, int mu, int sign,       \
                       int eqop, const int *idx_a, const int *gang);              \
void ora_rtimes_##SFX(R *r, R a, const R *b, long n, int ncplx, int eqop,        \
                      const int *idx_b, const int *gang);                         \
double ora_norm2_ref_##SFX(const R *a, long n, int ncplx, const int *idx_a,      \
                           const int *gang);                                      \
void ora_dot_ref_##SFX(double *out2, const R *a, const R *b, long n, int ncplx,  \
                       const int *idx_a, const int *idx_b, const int *gang);      \
void ora_dot_field_##SFX(R *r, const R *a, const R *b, long n, int ncplx,        \
                         const int *idx_a, const int *idx_b, const int *gang);    \
double ora_norm2_exact_##SFX(const R *a, long n, int ncplx, const int *idx_a,    \
                             const int *gang);                                    \
void ora_dot_exact_##SFX(double *out2, const R *a, const R *b, long n, int ncplx,\
                         const int *idx_a, const int *idx_b, const int *gang);                  \
void ora_prop_##SFX(int kind, int ca, int cb, int eqop, R *r, const R *a, const R *b,  \
                    long n, const int *idx_a, const int *idx_b, const int *gang);

ORA_DECL(f, float)
ORA_DECL(d, double)

/* matrix functions: which = ORA_MF_*; det writes one complex per site */
#define ORA_MF_EXP 0
#define ORA_MF_SQRT 1
#define ORA_MF_INVERSE 2
#define ORA_MF_DET 3
#define ORA_MF_INVSQRT 4
#define ORA_MF_LOG 5
#define ORA_MF_EXPA 6
#define ORA_MF_EXPTA 7
#define ORA_MF_SQRTPH 8
#define ORA_MF_INVSQRTPH 9
#define ORA_MF_EIGENVALS 10
#define ORA_MF_EIGENVALSH 11
int ora_mfunc_f(float *r, const float *a, long n, int nc, int which);
int ora_mfunc_d(double *r, const double *a, long n, int nc, int which);
/* r = a^-1 b per site; nb = 1 (ColorVector) or nc (ColorMatrix) */
void ora_minv_f(float *r, const float *a, const float *b, long n, int nc, int nb, const int *ia, const int *ib);
void ora_minv_d(double *r, const double *a, const double *b, long n, int nc, int nb, const int *ia,
                const int *ib);

/* element-wise families (shape / perm codes as the product's EwShape / EwPerm),
 * the ColorVector outer product and site-local dot products (kind as LdKind) */
void ora_ewise_f(int shape, int perm, int eqop, float *r, const float *b, const float *c, const float *s,
                 int scal_kind, float sre, float sim, long n, int ne, const int *idx_b, const int *idx_c,
                 const int *idx_s, const int *gang);
void ora_ewise_d(int shape, int perm, int eqop, double *r, const double *b, const double *c, const double *s,
                 int scal_kind, double sre, double sim, long n, int ne, const int *idx_b, const int *idx_c,
                 const int *idx_s, const int *gang);
void ora_outer_f(int eqop, float *r, const float *a, const float *b, long n, const int *idx_a, const int *idx_b,
                 const int *gang);
void ora_outer_d(int eqop, double *r, const double *a, const double *b, long n, const int *idx_a,
                 const int *idx_b, const int *gang);
void ora_ldot_f(int kind, int perm, int eqop, float *r, const float *a, const float *b, long n, int ne,
                const int *idx_a, const int *idx_b, const int *gang);
void ora_ldot_d(int kind, int perm, int eqop, double *r, const double *a, const double *b, long n, int ne,
                const int *idx_a, const int *idx_b, const int *gang);

/* QLA_I_ integer ops (codes as the product's IntCode, 19 = mask) */
void ora_int(int code, int eqop, int *r, const int *a, const int *b, const int *c, int s, long n,
             const int *ia, const int *ib, const int *ic, const int *gang);

/* site-field families: fills, copymask, components ('e', 'c', 'd'), gamma
 * multiplication, traces (kind 0 C, 1 Re, 2 Im, 3 antiherm), global
 * reductions of P / Ma / Pa in the reference order, global sums */
#define ORA_SITEFIELD_DECL(R, SFX)                                                               \
void ora_fill_##SFX(int eqop, R *r, const R *a, long n, int ne, const int *gang);                \
void ora_diagfill_##SFX(int eqop, R *r, const R *c, long n, const int *gang);                    \
void ora_zero_##SFX(R *r, long n, int ne, const int *gang);                                      \
void ora_mask_##SFX(R *r, const R *a, const int *m, long n, int ne, const int *idx_a,           \
                    const int *idx_m, const int *gang);                                           \
void ora_component_##SFX(int what, int dst, int src, R *r, const R *a, int i_c, int i_s,         \
                         int j_c, int j_s, long n, const int *idx_a, const int *gang);          \
void ora_gamma_##SFX(int right, int ne, int mu, R *r, const R *a, long n, const int *idx_a,      \
                     const int *gang);                                                            \
void ora_trace_##SFX(int kind, R *r, const R *a, long n, const int *idx_a, const int *gang);    \
void ora_gdot_##SFX(int kind, int perm, double *out2, const R *a, const R *b, long n, int ne,     \
                    const int *idx_a, const int *idx_b, const int *gang);                        \
void ora_gsum_##SFX(double *out, const R *a, long n, int ne, const int *idx_a, const int *gang);
ORA_SITEFIELD_DECL(float, f)
ORA_SITEFIELD_DECL(double, d)
/* the same families with the colour count nc as the first argument (the
 * QLA_FN_ / QLA_DN_ libraries) */
#define ORA_NCOLOR_DECL(R, SFX)                                                                   \
void ora_ewise_n_##SFX(int nc, int shape, int perm, int eqop, R *r, const R *b, const R *c,       \
                       const R *s, int scal_kind, R sre, R sim, long n, int ne, const int *idx_b, \
                       const int *idx_c, const int *idx_s, const int *gang);                     \
void ora_outer_n_##SFX(int nc, int eqop, R *r, const R *a, const R *b, long n, const int *idx_a,  \
                       const int *idx_b, const int *gang);                                       \
void ora_ldot_n_##SFX(int nc, int kind, int perm, int eqop, R *r, const R *a, const R *b, long n, \
                      int ne, const int *idx_a, const int *idx_b, const int *gang);              \
void ora_diagfill_n_##SFX(int nc, int eqop, R *r, const R *c, long n, const int *gang);          \
void ora_component_n_##SFX(int nc, int what, int dst, int src, R *r, const R *a, int i_c,         \
                           int i_s, int j_c, int j_s, long n, const int *idx_a, const int *gang); \
void ora_gamma_n_##SFX(int nc, int right, int ne, int mu, R *r, const R *a, long n,              \
                       const int *idx_a, const int *gang);                                       \
void ora_trace_n_##SFX(int nc, int kind, R *r, const R *a, long n, const int *idx_a,             \
                       const int *gang);                                                          \
void ora_gdot_n_##SFX(int nc, int kind, int perm, double *out2, const R *a, const R *b, long n,    \
                      int ne, const int *idx_a, const int *idx_b, const int *gang);
void ora_prop_n_f(int nc, int kind, int ca, int cb, int eqop, float *r, const float *a, const float *b, long n,
                  const int *idx_a, const int *idx_b, const int *gang);
void ora_prop_n_d(int nc, int kind, int ca, int cb, int eqop, double *r, const double *a, const double *b, long n,
                  const int *idx_a, const int *idx_b, const int *gang);
ORA_NCOLOR_DECL(float, f)
ORA_NCOLOR_DECL(double, d)
/* precision conversions of n records of nr reals: QLA_DF_c_eq_c (float to
 * double) and QLA_FD_c_eq_c (double to float, rounded to nearest) */
void ora_convert_df(double *r, const float *a, long n, int nr, const int *idx_a, const int *gang);
void ora_convert_fd(float *r, const double *a, long n, int nr, const int *idx_a, const int *gang);

/* the per-site random-number generator (state: 11 32-bit words) */
float ora_rng_uniform(void *state);
float ora_rng_gaussian(void *state, int milc);
void ora_rng_seed(void *state, int seed, int index);
void ora_rng_fill_f(int nreal, int gauss, int milc, float *r, void *s, long n, const int *idx_s, const int *gang);
void ora_rng_fill_d(int nreal, int gauss, int milc, double *r, void *s, long n, const int *idx_s, const int *gang);
void ora_rng_seedfield(void *r, int seed, const int *a, long n, const int *idx_a, const int *gang);
void ora_rng_copy(void *r, const void *a, const int *mask, long n, const int *idx_a, const int *idx_m,
                  const int *gang);

/* QLA_F_ / QLA_D_ real, complex and integer fields (op codes as the
 * product's ScalarOp) and the reference-order global sums of real / integer
 * fields (kind 0 dot, 1 norm2, 2 sum) */
void ora_scalar_f(int op, int eqop, void *r, const void *a, const void *b, const void *c, float s, long n,
                  const int *ia, const int *ib, const int *ic, const int *gang);
void ora_scalar_d(int op, int eqop, void *r, const void *a, const void *b, const void *c, double s, long n,
                  const int *ia, const int *ib, const int *ic, const int *gang);
double ora_sred_f(int kind, int isint, const void *a, const void *b, long n, const int *ia, const int *ib,
                  const int *gang);
double ora_sred_d(int kind, int isint, const void *a, const void *b, long n, const int *ia, const int *ib,
                  const int *gang);

int ora_version(void);

#endif
