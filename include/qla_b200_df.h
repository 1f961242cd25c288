/*
 * qla_b200_df.h -- GENERATED by qla_b200/gen/gen_qla.py; do not edit.
 *
 * QLA DF level-1 entry points implemented by libqla_b200.so (sm_100a).
 * Each declaration replaces the reference function of the same name, whose
 * C loop the reference generator emits from the cited section.  Array
 * arguments are device pointers; see qla_b200_runtime.h for scalars,
 * reduction outputs, streams and errors.
 */
#ifndef QLA_B200_DF_H
#define QLA_B200_DF_H
#include "qla_b200_types.h"

#ifdef __cplusplus
#define QLA_B200_RESTRICT __restrict__
extern "C" {
#else
#define QLA_B200_RESTRICT restrict
#endif

/* ---- sglobal: replaces the DF functions emitted by lib/perl/build_qla.pl:186-355 */
/* replaces QLA_DF_c_veq_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_c_veq_C_dot_C(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_DF_c_veq_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_c_veq_C_dot_pC(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_DF_c_veq_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_c_veq_pC_dot_C(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_DF_c_veq_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_c_veq_pC_dot_pC(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_DF_c_xeq_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_c_xeq_C_dot_C(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_DF_c_xeq_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_c_xeq_C_dot_pC(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_DF_c_xeq_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_c_xeq_pC_dot_C(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_DF_c_xeq_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_c_xeq_pC_dot_pC(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_DF_c_veq_Ca_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_c_veq_Ca_dot_C(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_DF_c_veq_Ca_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_c_veq_Ca_dot_pC(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_DF_c_veq_pCa_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_c_veq_pCa_dot_C(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_DF_c_veq_pCa_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_c_veq_pCa_dot_pC(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_DF_c_xeq_Ca_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_c_xeq_Ca_dot_C(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_DF_c_xeq_Ca_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_c_xeq_Ca_dot_pC(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_DF_c_xeq_pCa_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_c_xeq_pCa_dot_C(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_DF_c_xeq_pCa_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_c_xeq_pCa_dot_pC(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_DF_c_veq_sum_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_c_veq_sum_C(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_DF_c_veq_sum_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_c_veq_sum_pC(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_DF_c_xeq_sum_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_c_xeq_sum_C(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_DF_c_xeq_sum_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_c_xeq_sum_pC(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_DF_r_veq_R_dot_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_veq_R_dot_R(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_DF_r_veq_R_dot_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_veq_R_dot_pR(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_DF_r_veq_pR_dot_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_veq_pR_dot_R(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_DF_r_veq_pR_dot_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_veq_pR_dot_pR(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_DF_r_xeq_R_dot_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_xeq_R_dot_R(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_DF_r_xeq_R_dot_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_xeq_R_dot_pR(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_DF_r_xeq_pR_dot_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_xeq_pR_dot_R(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_DF_r_xeq_pR_dot_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_xeq_pR_dot_pR(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_DF_r_veq_norm2_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_veq_norm2_C(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_DF_r_veq_norm2_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_veq_norm2_pC(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_DF_r_xeq_norm2_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_xeq_norm2_C(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_DF_r_xeq_norm2_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_xeq_norm2_pC(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_DF_r_veq_norm2_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_veq_norm2_R(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_DF_r_veq_norm2_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_veq_norm2_pR(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_DF_r_xeq_norm2_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_xeq_norm2_R(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_DF_r_xeq_norm2_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_xeq_norm2_pR(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_DF_r_veq_re_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_veq_re_C_dot_C(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_DF_r_veq_re_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_veq_re_C_dot_pC(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_DF_r_veq_re_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_veq_re_pC_dot_C(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_DF_r_veq_re_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_veq_re_pC_dot_pC(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_DF_r_xeq_re_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_xeq_re_C_dot_C(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_DF_r_xeq_re_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_xeq_re_C_dot_pC(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_DF_r_xeq_re_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_xeq_re_pC_dot_C(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_DF_r_xeq_re_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_xeq_re_pC_dot_pC(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_DF_r_veq_sum_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_veq_sum_R(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_DF_r_veq_sum_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_veq_sum_pR(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_DF_r_xeq_sum_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_xeq_sum_R(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_DF_r_xeq_sum_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_r_xeq_sum_pR(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* ---- convert: replaces the DF functions emitted by lib/perl/build_qla.pl:186-355 */
/* replaces QLA_DF_R_veq_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_R_veq_R(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_FD_R_veq_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_FD_R_veq_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_D_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_DF_R_veq_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_R_veq_pR(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_FD_R_veq_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_FD_R_veq_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_D_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_DF_C_veq_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_C_veq_C(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_FD_C_veq_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_FD_C_veq_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_D_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_DF_C_veq_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_C_veq_pC(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_FD_C_veq_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_FD_C_veq_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_D_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_DF_R_xeq_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_R_xeq_R(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_FD_R_xeq_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_FD_R_xeq_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_D_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_DF_R_xeq_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_R_xeq_pR(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_FD_R_xeq_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_FD_R_xeq_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_D_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_DF_C_xeq_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_C_xeq_C(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_FD_C_xeq_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_FD_C_xeq_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_D_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_DF_C_xeq_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_DF_C_xeq_pC(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_FD_C_xeq_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_FD_C_xeq_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_D_Complex *QLA_B200_RESTRICT * a, int * index, int n);

#ifdef __cplusplus
}
#endif
#endif
