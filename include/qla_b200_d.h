/*
 * qla_b200_d.h -- GENERATED by qla_b200/gen/gen_qla.py; do not edit.
 *
 * QLA D level-1 entry points implemented by libqla_b200.so (sm_100a).
 * Each declaration replaces the reference function of the same name, whose
 * C loop the reference generator emits from the cited section.  Array
 * arguments are device pointers; see qla_b200_runtime.h for scalars,
 * reduction outputs, streams and errors.
 */
#ifndef QLA_B200_D_H
#define QLA_B200_D_H
#include "qla_b200_types.h"

#ifdef __cplusplus
#define QLA_B200_RESTRICT __restrict__
extern "C" {
#else
#define QLA_B200_RESTRICT restrict
#endif

/* ---- random: replaces the D functions emitted by lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills */
/* replaces QLA_D_R_veq_random_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_D_R_veq_random_S(QLA_D_Real *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT a, int n);
/* replaces QLA_D_R_veq_gaussian_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_D_R_veq_gaussian_S(QLA_D_Real *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT a, int n);
/* replaces QLA_D_C_veq_gaussian_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_D_C_veq_gaussian_S(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT a, int n);
/* replaces QLA_D_R_veq_random_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_D_R_veq_random_pS(QLA_D_Real *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_D_R_veq_gaussian_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_D_R_veq_gaussian_pS(QLA_D_Real *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_D_C_veq_gaussian_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_D_C_veq_gaussian_pS(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_D_R_xeq_random_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_D_R_xeq_random_S(QLA_D_Real *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_D_R_xeq_gaussian_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_D_R_xeq_gaussian_S(QLA_D_Real *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_D_C_xeq_gaussian_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_D_C_xeq_gaussian_S(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_D_R_xeq_random_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_D_R_xeq_random_pS(QLA_D_Real *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_D_R_xeq_gaussian_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_D_R_xeq_gaussian_pS(QLA_D_Real *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_D_C_xeq_gaussian_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_D_C_xeq_gaussian_pS(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT * a, int * index, int n);

#ifdef __cplusplus
}
#endif
#endif
