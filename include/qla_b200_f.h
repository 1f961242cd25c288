/*
 * qla_b200_f.h -- GENERATED by qla_b200/gen/gen_qla.py; do not edit.
 *
 * QLA F level-1 entry points implemented by libqla_b200.so (sm_100a).
 * Each declaration replaces the reference function of the same name, whose
 * C loop the reference generator emits from the cited section.  Array
 * arguments are device pointers; see qla_b200_runtime.h for scalars,
 * reduction outputs, streams and errors.
 */
#ifndef QLA_B200_F_H
#define QLA_B200_F_H
#include "qla_b200_types.h"

#ifdef __cplusplus
#define QLA_B200_RESTRICT __restrict__
extern "C" {
#else
#define QLA_B200_RESTRICT restrict
#endif

/* ---- cfield: replaces the F functions emitted by lib/perl/build_qla.pl:186-355 */
/* replaces QLA_F_C_veq_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_C_veq_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_C_vpeq_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_C_vpeq_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_C_vmeq_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_C_vmeq_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_C_veqm_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_C_veqm_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_C_xeq_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_C_xeq_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_C_xpeq_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_C_xpeq_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_C_xmeq_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_C_xmeq_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_C_xeqm_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_C_xeqm_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_C_veq_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_C_veq_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_C_vpeq_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_C_vpeq_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_C_vmeq_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_C_vmeq_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_C_veqm_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_C_veqm_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_C_xeq_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_C_xeq_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_C_xpeq_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_C_xpeq_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_C_xmeq_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_C_xmeq_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_C_xeqm_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_C_xeqm_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_C_veq_i_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_i_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_C_veq_i_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_i_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_C_vpeq_i_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_i_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_C_vpeq_i_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_i_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_C_vmeq_i_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_i_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_C_vmeq_i_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_i_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_C_veqm_i_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_i_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_C_veqm_i_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_i_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_C_xeq_i_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_i_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_C_xeq_i_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_i_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_C_xpeq_i_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_i_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_C_xpeq_i_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_i_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_C_xmeq_i_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_i_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_C_xmeq_i_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_i_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_C_xeqm_i_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_i_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_C_xeqm_i_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_i_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_C_veq_c (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_c(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_C_vpeq_c (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_c(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_C_vmeq_c (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_c(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_C_veqm_c (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_c(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_C_xeq_c (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_c(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_C_xpeq_c (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_c(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_C_xmeq_c (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_c(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_C_xeqm_c (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_c(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_C_veq_zero (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_zero(QLA_F_Complex *QLA_B200_RESTRICT r, int n);
/* replaces QLA_F_C_xeq_zero (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_zero(QLA_F_Complex *QLA_B200_RESTRICT r, int * index, int n);
/* replaces QLA_F_C_veq_C_mask_I (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_C_mask_I(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_C_mask_pI (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_C_mask_pI(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veq_pC_mask_I (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pC_mask_I(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_pC_mask_pI (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pC_mask_pI(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_xeq_C_mask_I (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_C_mask_I(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_C_mask_pI (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_C_mask_pI(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeq_pC_mask_I (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pC_mask_I(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_pC_mask_pI (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pC_mask_pI(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_veq_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_R(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_C_veq_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pR(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_C_xeq_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_R(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_C_xeq_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pR(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_C_veq_R_plus_i_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_R_plus_i_R(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_R_plus_i_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_R_plus_i_pR(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veq_pR_plus_i_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pR_plus_i_R(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_pR_plus_i_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pR_plus_i_pR(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_xeq_R_plus_i_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_R_plus_i_R(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_R_plus_i_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_R_plus_i_pR(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeq_pR_plus_i_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pR_plus_i_R(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_pR_plus_i_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pR_plus_i_pR(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_veq_C_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_C_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_C_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_C_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veq_pC_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pC_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_pC_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pC_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vpeq_C_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_C_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vpeq_C_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_C_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vpeq_pC_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_pC_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vpeq_pC_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_pC_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vmeq_C_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_C_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vmeq_C_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_C_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vmeq_pC_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_pC_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vmeq_pC_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_pC_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veqm_C_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_C_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veqm_C_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_C_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veqm_pC_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_pC_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veqm_pC_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_pC_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_xeq_C_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_C_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_C_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_C_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeq_pC_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pC_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_pC_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pC_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xpeq_C_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_C_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xpeq_C_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_C_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xpeq_pC_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_pC_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xpeq_pC_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_pC_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xmeq_C_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_C_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xmeq_C_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_C_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xmeq_pC_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_pC_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xmeq_pC_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_pC_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeqm_C_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_C_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeqm_C_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_C_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeqm_pC_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_pC_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeqm_pC_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_pC_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_veq_C_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_C_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_C_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_C_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veq_pC_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pC_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_pC_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pC_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vpeq_C_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_C_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vpeq_C_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_C_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vpeq_pC_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_pC_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vpeq_pC_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_pC_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vmeq_C_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_C_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vmeq_C_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_C_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vmeq_pC_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_pC_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vmeq_pC_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_pC_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veqm_C_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_C_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veqm_C_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_C_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veqm_pC_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_pC_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veqm_pC_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_pC_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_xeq_C_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_C_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_C_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_C_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeq_pC_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pC_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_pC_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pC_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xpeq_C_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_C_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xpeq_C_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_C_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xpeq_pC_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_pC_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xpeq_pC_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_pC_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xmeq_C_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_C_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xmeq_C_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_C_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xmeq_pC_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_pC_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xmeq_pC_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_pC_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeqm_C_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_C_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeqm_C_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_C_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeqm_pC_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_pC_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeqm_pC_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_pC_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_veq_Ca_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_Ca_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_Ca_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_Ca_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veq_pCa_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pCa_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_pCa_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pCa_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vpeq_Ca_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_Ca_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vpeq_Ca_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_Ca_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vpeq_pCa_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_pCa_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vpeq_pCa_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_pCa_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vmeq_Ca_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_Ca_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vmeq_Ca_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_Ca_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vmeq_pCa_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_pCa_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vmeq_pCa_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_pCa_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veqm_Ca_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_Ca_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veqm_Ca_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_Ca_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veqm_pCa_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_pCa_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veqm_pCa_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_pCa_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_xeq_Ca_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_Ca_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_Ca_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_Ca_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeq_pCa_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pCa_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_pCa_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pCa_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xpeq_Ca_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_Ca_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xpeq_Ca_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_Ca_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xpeq_pCa_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_pCa_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xpeq_pCa_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_pCa_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xmeq_Ca_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_Ca_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xmeq_Ca_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_Ca_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xmeq_pCa_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_pCa_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xmeq_pCa_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_pCa_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeqm_Ca_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_Ca_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeqm_Ca_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_Ca_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeqm_pCa_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_pCa_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeqm_pCa_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_pCa_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_veq_Ca_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_Ca_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_Ca_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_Ca_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veq_pCa_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pCa_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_pCa_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pCa_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vpeq_Ca_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_Ca_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vpeq_Ca_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_Ca_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vpeq_pCa_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_pCa_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vpeq_pCa_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_pCa_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vmeq_Ca_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_Ca_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vmeq_Ca_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_Ca_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vmeq_pCa_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_pCa_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vmeq_pCa_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_pCa_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veqm_Ca_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_Ca_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veqm_Ca_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_Ca_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veqm_pCa_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_pCa_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veqm_pCa_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_pCa_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_xeq_Ca_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_Ca_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_Ca_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_Ca_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeq_pCa_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pCa_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_pCa_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pCa_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xpeq_Ca_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_Ca_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xpeq_Ca_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_Ca_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xpeq_pCa_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_pCa_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xpeq_pCa_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_pCa_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xmeq_Ca_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_Ca_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xmeq_Ca_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_Ca_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xmeq_pCa_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_pCa_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xmeq_pCa_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_pCa_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeqm_Ca_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_Ca_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeqm_Ca_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_Ca_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeqm_pCa_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_pCa_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeqm_pCa_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_pCa_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_veq_R_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_R_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_R_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_R_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veq_pR_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pR_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_pR_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pR_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vpeq_R_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_R_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vpeq_R_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_R_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vpeq_pR_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_pR_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vpeq_pR_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_pR_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vmeq_R_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_R_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vmeq_R_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_R_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vmeq_pR_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_pR_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vmeq_pR_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_pR_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veqm_R_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_R_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veqm_R_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_R_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veqm_pR_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_pR_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veqm_pR_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_pR_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_xeq_R_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_R_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_R_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_R_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeq_pR_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pR_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_pR_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pR_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xpeq_R_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_R_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xpeq_R_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_R_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xpeq_pR_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_pR_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xpeq_pR_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_pR_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xmeq_R_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_R_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xmeq_R_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_R_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xmeq_pR_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_pR_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xmeq_pR_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_pR_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeqm_R_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_R_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeqm_R_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_R_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeqm_pR_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_pR_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeqm_pR_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_pR_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_veq_R_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_R_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_R_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_R_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veq_pR_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pR_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_pR_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pR_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vpeq_R_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_R_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vpeq_R_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_R_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vpeq_pR_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_pR_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vpeq_pR_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_pR_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vmeq_R_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_R_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vmeq_R_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_R_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vmeq_pR_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_pR_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vmeq_pR_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_pR_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veqm_R_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_R_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veqm_R_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_R_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veqm_pR_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_pR_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veqm_pR_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_pR_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_xeq_R_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_R_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_R_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_R_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeq_pR_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pR_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_pR_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pR_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xpeq_R_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_R_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xpeq_R_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_R_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xpeq_pR_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_pR_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xpeq_pR_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_pR_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xmeq_R_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_R_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xmeq_R_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_R_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xmeq_pR_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_pR_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xmeq_pR_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_pR_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeqm_R_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_R_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeqm_R_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_R_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeqm_pR_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_pR_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeqm_pR_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_pR_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_veq_c_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_c_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_c_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_c_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vpeq_c_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_c_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vpeq_c_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_c_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vmeq_c_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_c_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vmeq_c_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_c_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veqm_c_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_c_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veqm_c_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_c_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_xeq_c_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_c_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_c_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_c_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xpeq_c_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_c_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xpeq_c_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_c_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xmeq_c_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_c_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xmeq_c_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_c_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeqm_c_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_c_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeqm_c_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_c_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_veq_c_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_c_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_c_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_c_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vpeq_c_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_c_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vpeq_c_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_c_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vmeq_c_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_c_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vmeq_c_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_c_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veqm_c_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_c_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veqm_c_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_c_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_xeq_c_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_c_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_c_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_c_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xpeq_c_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_c_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xpeq_c_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_c_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xmeq_c_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_c_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xmeq_c_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_c_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeqm_c_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_c_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeqm_c_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_c_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_veq_r_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_r_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_r_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_r_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vpeq_r_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_r_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vpeq_r_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_r_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vmeq_r_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_r_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vmeq_r_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_r_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veqm_r_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_r_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veqm_r_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_r_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_xeq_r_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_r_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_r_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_r_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xpeq_r_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_r_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xpeq_r_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_r_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xmeq_r_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_r_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xmeq_r_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_r_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeqm_r_times_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_r_times_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeqm_r_times_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_r_times_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_veq_r_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_r_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_r_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_r_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vpeq_r_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_r_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vpeq_r_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_r_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vmeq_r_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_r_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vmeq_r_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_r_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veqm_r_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_r_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veqm_r_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_r_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_xeq_r_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_r_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_r_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_r_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xpeq_r_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_r_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xpeq_r_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_r_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xmeq_r_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_r_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xmeq_r_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_r_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeqm_r_times_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_r_times_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeqm_r_times_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_r_times_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_veq_C_plus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_C_plus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_C_plus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_C_plus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veq_pC_plus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pC_plus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_pC_plus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pC_plus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_xeq_C_plus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_C_plus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_C_plus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_C_plus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeq_pC_plus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pC_plus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_pC_plus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pC_plus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_veq_C_minus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_C_minus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_C_minus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_C_minus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veq_pC_minus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pC_minus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_pC_minus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pC_minus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_xeq_C_minus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_C_minus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_C_minus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_C_minus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeq_pC_minus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pC_minus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_pC_minus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pC_minus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_veq_c_times_C_plus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_c_times_C_plus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, QLA_F_Complex *QLA_B200_RESTRICT c, int n);
/* replaces QLA_F_C_veq_c_times_C_plus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_c_times_C_plus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, QLA_F_Complex *QLA_B200_RESTRICT * c, int n);
/* replaces QLA_F_C_veq_c_times_pC_plus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_c_times_pC_plus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, QLA_F_Complex *QLA_B200_RESTRICT c, int n);
/* replaces QLA_F_C_veq_c_times_pC_plus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_c_times_pC_plus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, QLA_F_Complex *QLA_B200_RESTRICT * c, int n);
/* replaces QLA_F_C_xeq_c_times_C_plus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_c_times_C_plus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, QLA_F_Complex *QLA_B200_RESTRICT c, int * index, int n);
/* replaces QLA_F_C_xeq_c_times_C_plus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_c_times_C_plus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, QLA_F_Complex *QLA_B200_RESTRICT * c, int * index, int n);
/* replaces QLA_F_C_xeq_c_times_pC_plus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_c_times_pC_plus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, QLA_F_Complex *QLA_B200_RESTRICT c, int * index, int n);
/* replaces QLA_F_C_xeq_c_times_pC_plus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_c_times_pC_plus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, QLA_F_Complex *QLA_B200_RESTRICT * c, int * index, int n);
/* replaces QLA_F_C_veq_c_times_C_minus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_c_times_C_minus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, QLA_F_Complex *QLA_B200_RESTRICT c, int n);
/* replaces QLA_F_C_veq_c_times_C_minus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_c_times_C_minus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, QLA_F_Complex *QLA_B200_RESTRICT * c, int n);
/* replaces QLA_F_C_veq_c_times_pC_minus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_c_times_pC_minus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, QLA_F_Complex *QLA_B200_RESTRICT c, int n);
/* replaces QLA_F_C_veq_c_times_pC_minus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_c_times_pC_minus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, QLA_F_Complex *QLA_B200_RESTRICT * c, int n);
/* replaces QLA_F_C_xeq_c_times_C_minus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_c_times_C_minus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, QLA_F_Complex *QLA_B200_RESTRICT c, int * index, int n);
/* replaces QLA_F_C_xeq_c_times_C_minus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_c_times_C_minus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, QLA_F_Complex *QLA_B200_RESTRICT * c, int * index, int n);
/* replaces QLA_F_C_xeq_c_times_pC_minus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_c_times_pC_minus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, QLA_F_Complex *QLA_B200_RESTRICT c, int * index, int n);
/* replaces QLA_F_C_xeq_c_times_pC_minus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_c_times_pC_minus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, QLA_F_Complex *QLA_B200_RESTRICT * c, int * index, int n);
/* replaces QLA_F_C_veq_r_times_C_plus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_r_times_C_plus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, QLA_F_Complex *QLA_B200_RESTRICT c, int n);
/* replaces QLA_F_C_veq_r_times_C_plus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_r_times_C_plus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, QLA_F_Complex *QLA_B200_RESTRICT * c, int n);
/* replaces QLA_F_C_veq_r_times_pC_plus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_r_times_pC_plus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, QLA_F_Complex *QLA_B200_RESTRICT c, int n);
/* replaces QLA_F_C_veq_r_times_pC_plus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_r_times_pC_plus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, QLA_F_Complex *QLA_B200_RESTRICT * c, int n);
/* replaces QLA_F_C_xeq_r_times_C_plus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_r_times_C_plus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, QLA_F_Complex *QLA_B200_RESTRICT c, int * index, int n);
/* replaces QLA_F_C_xeq_r_times_C_plus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_r_times_C_plus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, QLA_F_Complex *QLA_B200_RESTRICT * c, int * index, int n);
/* replaces QLA_F_C_xeq_r_times_pC_plus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_r_times_pC_plus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, QLA_F_Complex *QLA_B200_RESTRICT c, int * index, int n);
/* replaces QLA_F_C_xeq_r_times_pC_plus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_r_times_pC_plus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, QLA_F_Complex *QLA_B200_RESTRICT * c, int * index, int n);
/* replaces QLA_F_C_veq_r_times_C_minus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_r_times_C_minus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, QLA_F_Complex *QLA_B200_RESTRICT c, int n);
/* replaces QLA_F_C_veq_r_times_C_minus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_r_times_C_minus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, QLA_F_Complex *QLA_B200_RESTRICT * c, int n);
/* replaces QLA_F_C_veq_r_times_pC_minus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_r_times_pC_minus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, QLA_F_Complex *QLA_B200_RESTRICT c, int n);
/* replaces QLA_F_C_veq_r_times_pC_minus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_r_times_pC_minus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, QLA_F_Complex *QLA_B200_RESTRICT * c, int n);
/* replaces QLA_F_C_xeq_r_times_C_minus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_r_times_C_minus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, QLA_F_Complex *QLA_B200_RESTRICT c, int * index, int n);
/* replaces QLA_F_C_xeq_r_times_C_minus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_r_times_C_minus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, QLA_F_Complex *QLA_B200_RESTRICT * c, int * index, int n);
/* replaces QLA_F_C_xeq_r_times_pC_minus_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_r_times_pC_minus_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, QLA_F_Complex *QLA_B200_RESTRICT c, int * index, int n);
/* replaces QLA_F_C_xeq_r_times_pC_minus_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_r_times_pC_minus_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, QLA_F_Complex *QLA_B200_RESTRICT * c, int * index, int n);
/* replaces QLA_F_C_veq_C_divide_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_C_divide_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_C_divide_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_C_divide_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veq_pC_divide_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pC_divide_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_pC_divide_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pC_divide_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_xeq_C_divide_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_C_divide_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_C_divide_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_C_divide_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeq_pC_divide_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pC_divide_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_pC_divide_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pC_divide_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_veq_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_C_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_C_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veq_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pC_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pC_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vpeq_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_C_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vpeq_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_C_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vpeq_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_pC_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vpeq_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_pC_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vmeq_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_C_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vmeq_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_C_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vmeq_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_pC_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vmeq_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_pC_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veqm_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_C_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veqm_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_C_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veqm_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_pC_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veqm_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_pC_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_xeq_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_C_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_C_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeq_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pC_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pC_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xpeq_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_C_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xpeq_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_C_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xpeq_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_pC_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xpeq_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_pC_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xmeq_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_C_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xmeq_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_C_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xmeq_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_pC_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xmeq_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_pC_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeqm_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_C_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeqm_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_C_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeqm_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_pC_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeqm_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_pC_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_veq_C_dot_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_C_dot_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_C_dot_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_C_dot_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veq_pC_dot_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pC_dot_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_pC_dot_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pC_dot_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vpeq_C_dot_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_C_dot_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vpeq_C_dot_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_C_dot_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vpeq_pC_dot_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_pC_dot_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vpeq_pC_dot_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_pC_dot_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vmeq_C_dot_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_C_dot_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vmeq_C_dot_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_C_dot_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vmeq_pC_dot_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_pC_dot_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vmeq_pC_dot_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_pC_dot_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veqm_C_dot_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_C_dot_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veqm_C_dot_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_C_dot_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veqm_pC_dot_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_pC_dot_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veqm_pC_dot_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_pC_dot_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_xeq_C_dot_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_C_dot_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_C_dot_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_C_dot_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeq_pC_dot_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pC_dot_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_pC_dot_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pC_dot_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xpeq_C_dot_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_C_dot_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xpeq_C_dot_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_C_dot_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xpeq_pC_dot_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_pC_dot_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xpeq_pC_dot_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_pC_dot_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xmeq_C_dot_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_C_dot_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xmeq_C_dot_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_C_dot_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xmeq_pC_dot_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_pC_dot_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xmeq_pC_dot_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_pC_dot_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeqm_C_dot_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_C_dot_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeqm_C_dot_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_C_dot_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeqm_pC_dot_Ca (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_pC_dot_Ca(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeqm_pC_dot_pCa (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_pC_dot_pCa(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_veq_Ca_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_Ca_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_Ca_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_Ca_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veq_pCa_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pCa_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veq_pCa_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_pCa_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vpeq_Ca_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_Ca_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vpeq_Ca_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_Ca_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vpeq_pCa_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_pCa_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vpeq_pCa_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vpeq_pCa_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vmeq_Ca_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_Ca_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vmeq_Ca_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_Ca_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_vmeq_pCa_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_pCa_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_vmeq_pCa_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_vmeq_pCa_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veqm_Ca_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_Ca_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veqm_Ca_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_Ca_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_veqm_pCa_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_pCa_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_C_veqm_pCa_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veqm_pCa_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_C_xeq_Ca_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_Ca_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_Ca_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_Ca_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeq_pCa_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pCa_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeq_pCa_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_pCa_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xpeq_Ca_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_Ca_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xpeq_Ca_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_Ca_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xpeq_pCa_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_pCa_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xpeq_pCa_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xpeq_pCa_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xmeq_Ca_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_Ca_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xmeq_Ca_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_Ca_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xmeq_pCa_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_pCa_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xmeq_pCa_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xmeq_pCa_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeqm_Ca_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_Ca_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeqm_Ca_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_Ca_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_xeqm_pCa_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_pCa_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_C_xeqm_pCa_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeqm_pCa_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_C_veq_cexp_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_cexp_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_C_veq_cexp_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_cexp_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_C_xeq_cexp_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_cexp_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_C_xeq_cexp_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_cexp_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_C_veq_clog_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_clog_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_C_veq_clog_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_clog_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_C_xeq_clog_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_clog_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_C_xeq_clog_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_clog_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_C_veq_csqrt_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_csqrt_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_C_veq_csqrt_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_csqrt_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_C_xeq_csqrt_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_csqrt_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_C_xeq_csqrt_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_csqrt_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_C_veq_cexpi_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_cexpi_R(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_C_veq_cexpi_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_veq_cexpi_pR(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_C_xeq_cexpi_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_cexpi_R(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_C_xeq_cexpi_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_C_xeq_cexpi_pR(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* ---- rfield: replaces the F functions emitted by lib/perl/build_qla.pl:186-355 */
/* replaces QLA_F_R_veq_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_vpeq_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vpeq_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_vpeq_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vpeq_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_vmeq_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vmeq_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_vmeq_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vmeq_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_veqm_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veqm_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veqm_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veqm_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_xpeq_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xpeq_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xpeq_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xpeq_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_xmeq_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xmeq_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xmeq_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xmeq_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_xeqm_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeqm_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeqm_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeqm_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_veq_I (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_I(QLA_F_Real *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_pI (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pI(QLA_F_Real *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_I (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_I(QLA_F_Real *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_pI (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pI(QLA_F_Real *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_veq_r (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_r(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_vpeq_r (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vpeq_r(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_vmeq_r (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vmeq_r(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veqm_r (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veqm_r(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_xeq_r (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_r(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xpeq_r (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xpeq_r(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xmeq_r (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xmeq_r(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeqm_r (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeqm_r(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_veq_zero (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_zero(QLA_F_Real *QLA_B200_RESTRICT r, int n);
/* replaces QLA_F_R_xeq_zero (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_zero(QLA_F_Real *QLA_B200_RESTRICT r, int * index, int n);
/* replaces QLA_F_R_veq_R_mask_I (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_R_mask_I(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_R_mask_pI (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_R_mask_pI(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_veq_pR_mask_I (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pR_mask_I(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_pR_mask_pI (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pR_mask_pI(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_xeq_R_mask_I (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_R_mask_I(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_R_mask_pI (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_R_mask_pI(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xeq_pR_mask_I (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pR_mask_I(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_pR_mask_pI (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pR_mask_pI(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_veq_R_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_R_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_R_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_R_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_veq_pR_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pR_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_pR_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pR_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_vpeq_R_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vpeq_R_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_vpeq_R_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vpeq_R_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_vpeq_pR_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vpeq_pR_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_vpeq_pR_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vpeq_pR_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_vmeq_R_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vmeq_R_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_vmeq_R_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vmeq_R_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_vmeq_pR_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vmeq_pR_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_vmeq_pR_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vmeq_pR_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_veqm_R_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veqm_R_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veqm_R_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veqm_R_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_veqm_pR_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veqm_pR_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veqm_pR_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veqm_pR_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_xeq_R_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_R_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_R_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_R_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xeq_pR_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pR_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_pR_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pR_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xpeq_R_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xpeq_R_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xpeq_R_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xpeq_R_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xpeq_pR_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xpeq_pR_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xpeq_pR_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xpeq_pR_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xmeq_R_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xmeq_R_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xmeq_R_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xmeq_R_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xmeq_pR_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xmeq_pR_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xmeq_pR_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xmeq_pR_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xeqm_R_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeqm_R_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeqm_R_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeqm_R_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xeqm_pR_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeqm_pR_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeqm_pR_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeqm_pR_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_veq_r_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_r_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_r_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_r_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_vpeq_r_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vpeq_r_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_vpeq_r_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vpeq_r_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_vmeq_r_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vmeq_r_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_vmeq_r_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vmeq_r_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_veqm_r_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veqm_r_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veqm_r_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veqm_r_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_xeq_r_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_r_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_r_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_r_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xpeq_r_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xpeq_r_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xpeq_r_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xpeq_r_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xmeq_r_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xmeq_r_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xmeq_r_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xmeq_r_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xeqm_r_times_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeqm_r_times_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeqm_r_times_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeqm_r_times_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_veq_r_times_R_plus_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_r_times_R_plus_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, QLA_F_Real *QLA_B200_RESTRICT c, int n);
/* replaces QLA_F_R_veq_r_times_R_plus_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_r_times_R_plus_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, QLA_F_Real *QLA_B200_RESTRICT * c, int n);
/* replaces QLA_F_R_veq_r_times_pR_plus_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_r_times_pR_plus_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, QLA_F_Real *QLA_B200_RESTRICT c, int n);
/* replaces QLA_F_R_veq_r_times_pR_plus_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_r_times_pR_plus_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, QLA_F_Real *QLA_B200_RESTRICT * c, int n);
/* replaces QLA_F_R_xeq_r_times_R_plus_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_r_times_R_plus_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, QLA_F_Real *QLA_B200_RESTRICT c, int * index, int n);
/* replaces QLA_F_R_xeq_r_times_R_plus_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_r_times_R_plus_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, QLA_F_Real *QLA_B200_RESTRICT * c, int * index, int n);
/* replaces QLA_F_R_xeq_r_times_pR_plus_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_r_times_pR_plus_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, QLA_F_Real *QLA_B200_RESTRICT c, int * index, int n);
/* replaces QLA_F_R_xeq_r_times_pR_plus_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_r_times_pR_plus_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, QLA_F_Real *QLA_B200_RESTRICT * c, int * index, int n);
/* replaces QLA_F_R_veq_r_times_R_minus_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_r_times_R_minus_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, QLA_F_Real *QLA_B200_RESTRICT c, int n);
/* replaces QLA_F_R_veq_r_times_R_minus_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_r_times_R_minus_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, QLA_F_Real *QLA_B200_RESTRICT * c, int n);
/* replaces QLA_F_R_veq_r_times_pR_minus_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_r_times_pR_minus_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, QLA_F_Real *QLA_B200_RESTRICT c, int n);
/* replaces QLA_F_R_veq_r_times_pR_minus_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_r_times_pR_minus_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, QLA_F_Real *QLA_B200_RESTRICT * c, int n);
/* replaces QLA_F_R_xeq_r_times_R_minus_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_r_times_R_minus_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, QLA_F_Real *QLA_B200_RESTRICT c, int * index, int n);
/* replaces QLA_F_R_xeq_r_times_R_minus_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_r_times_R_minus_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, QLA_F_Real *QLA_B200_RESTRICT * c, int * index, int n);
/* replaces QLA_F_R_xeq_r_times_pR_minus_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_r_times_pR_minus_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, QLA_F_Real *QLA_B200_RESTRICT c, int * index, int n);
/* replaces QLA_F_R_xeq_r_times_pR_minus_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_r_times_pR_minus_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, QLA_F_Real *QLA_B200_RESTRICT * c, int * index, int n);
/* replaces QLA_F_R_veq_R_ldexp_I (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_R_ldexp_I(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_R_ldexp_pI (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_R_ldexp_pI(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_veq_pR_ldexp_I (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pR_ldexp_I(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_pR_ldexp_pI (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pR_ldexp_pI(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_xeq_R_ldexp_I (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_R_ldexp_I(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_R_ldexp_pI (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_R_ldexp_pI(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xeq_pR_ldexp_I (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pR_ldexp_I(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_pR_ldexp_pI (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pR_ldexp_pI(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_veq_R_plus_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_R_plus_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_R_plus_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_R_plus_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_veq_pR_plus_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pR_plus_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_pR_plus_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pR_plus_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_xeq_R_plus_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_R_plus_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_R_plus_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_R_plus_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xeq_pR_plus_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pR_plus_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_pR_plus_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pR_plus_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_veq_R_minus_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_R_minus_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_R_minus_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_R_minus_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_veq_pR_minus_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pR_minus_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_pR_minus_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pR_minus_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_xeq_R_minus_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_R_minus_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_R_minus_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_R_minus_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xeq_pR_minus_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pR_minus_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_pR_minus_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pR_minus_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_veq_R_divide_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_R_divide_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_R_divide_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_R_divide_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_veq_pR_divide_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pR_divide_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_pR_divide_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pR_divide_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_xeq_R_divide_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_R_divide_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_R_divide_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_R_divide_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xeq_pR_divide_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pR_divide_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_pR_divide_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pR_divide_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_veq_R_max_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_R_max_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_R_max_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_R_max_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_veq_pR_max_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pR_max_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_pR_max_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pR_max_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_xeq_R_max_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_R_max_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_R_max_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_R_max_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xeq_pR_max_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pR_max_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_pR_max_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pR_max_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_veq_R_min_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_R_min_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_R_min_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_R_min_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_veq_pR_min_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pR_min_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_pR_min_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pR_min_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_xeq_R_min_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_R_min_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_R_min_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_R_min_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xeq_pR_min_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pR_min_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_pR_min_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pR_min_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_veq_R_mod_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_R_mod_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_R_mod_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_R_mod_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_veq_pR_mod_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pR_mod_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_pR_mod_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pR_mod_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_xeq_R_mod_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_R_mod_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_R_mod_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_R_mod_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xeq_pR_mod_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pR_mod_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_pR_mod_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pR_mod_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_veq_R_pow_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_R_pow_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_R_pow_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_R_pow_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_veq_pR_pow_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pR_pow_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_pR_pow_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pR_pow_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_xeq_R_pow_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_R_pow_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_R_pow_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_R_pow_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xeq_pR_pow_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pR_pow_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_pR_pow_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pR_pow_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_veq_R_atan2_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_R_atan2_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_R_atan2_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_R_atan2_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_veq_pR_atan2_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pR_atan2_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_pR_atan2_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_pR_atan2_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_xeq_R_atan2_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_R_atan2_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_R_atan2_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_R_atan2_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xeq_pR_atan2_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pR_atan2_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_pR_atan2_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_pR_atan2_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_veq_sin_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_sin_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_sin_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_sin_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_sin_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_sin_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_sin_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_sin_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_veq_cos_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_cos_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_cos_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_cos_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_cos_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_cos_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_cos_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_cos_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_veq_tan_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_tan_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_tan_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_tan_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_tan_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_tan_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_tan_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_tan_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_veq_asin_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_asin_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_asin_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_asin_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_asin_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_asin_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_asin_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_asin_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_veq_acos_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_acos_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_acos_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_acos_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_acos_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_acos_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_acos_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_acos_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_veq_atan_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_atan_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_atan_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_atan_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_atan_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_atan_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_atan_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_atan_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_veq_sqrt_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_sqrt_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_sqrt_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_sqrt_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_sqrt_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_sqrt_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_sqrt_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_sqrt_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_veq_fabs_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_fabs_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_fabs_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_fabs_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_fabs_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_fabs_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_fabs_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_fabs_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_veq_exp_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_exp_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_exp_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_exp_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_exp_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_exp_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_exp_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_exp_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_veq_log_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_log_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_log_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_log_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_log_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_log_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_log_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_log_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_veq_log10_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_log10_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_log10_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_log10_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_log10_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_log10_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_log10_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_log10_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_veq_sinh_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_sinh_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_sinh_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_sinh_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_sinh_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_sinh_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_sinh_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_sinh_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_veq_cosh_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_cosh_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_cosh_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_cosh_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_cosh_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_cosh_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_cosh_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_cosh_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_veq_tanh_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_tanh_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_tanh_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_tanh_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_tanh_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_tanh_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_tanh_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_tanh_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_veq_ceil_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_ceil_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_ceil_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_ceil_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_ceil_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_ceil_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_ceil_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_ceil_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_veq_floor_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_floor_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_floor_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_floor_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_floor_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_floor_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_floor_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_floor_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_veq_sign_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_sign_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_sign_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_sign_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_sign_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_sign_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_sign_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_sign_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_veq_re_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_re_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_re_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_re_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_re_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_re_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_re_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_re_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_veq_im_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_im_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_im_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_im_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_im_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_im_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_im_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_im_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_veq_norm_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_norm_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_norm_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_norm_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_norm_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_norm_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_norm_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_norm_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_veq_arg_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_arg_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_arg_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_arg_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_arg_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_arg_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_arg_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_arg_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* ---- cfield: replaces the F functions emitted by lib/perl/build_qla.pl:186-355 */
/* replaces QLA_F_R_veq_norm2_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_norm2_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_norm2_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_norm2_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_vpeq_norm2_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vpeq_norm2_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_vpeq_norm2_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vpeq_norm2_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_vmeq_norm2_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vmeq_norm2_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_vmeq_norm2_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vmeq_norm2_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_veqm_norm2_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veqm_norm2_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veqm_norm2_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veqm_norm2_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_norm2_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_norm2_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_norm2_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_norm2_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_xpeq_norm2_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xpeq_norm2_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xpeq_norm2_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xpeq_norm2_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_xmeq_norm2_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xmeq_norm2_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xmeq_norm2_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xmeq_norm2_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_xeqm_norm2_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeqm_norm2_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeqm_norm2_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeqm_norm2_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_veq_re_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_re_C_dot_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_re_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_re_C_dot_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_veq_re_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_re_pC_dot_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veq_re_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veq_re_pC_dot_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_vpeq_re_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vpeq_re_C_dot_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_vpeq_re_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vpeq_re_C_dot_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_vpeq_re_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vpeq_re_pC_dot_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_vpeq_re_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vpeq_re_pC_dot_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_vmeq_re_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vmeq_re_C_dot_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_vmeq_re_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vmeq_re_C_dot_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_vmeq_re_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vmeq_re_pC_dot_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_vmeq_re_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_vmeq_re_pC_dot_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_veqm_re_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veqm_re_C_dot_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veqm_re_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veqm_re_C_dot_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_veqm_re_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veqm_re_pC_dot_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_R_veqm_re_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_veqm_re_pC_dot_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_R_xeq_re_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_re_C_dot_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_re_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_re_C_dot_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xeq_re_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_re_pC_dot_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeq_re_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeq_re_pC_dot_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xpeq_re_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xpeq_re_C_dot_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xpeq_re_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xpeq_re_C_dot_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xpeq_re_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xpeq_re_pC_dot_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xpeq_re_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xpeq_re_pC_dot_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xmeq_re_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xmeq_re_C_dot_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xmeq_re_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xmeq_re_C_dot_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xmeq_re_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xmeq_re_pC_dot_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xmeq_re_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xmeq_re_pC_dot_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xeqm_re_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeqm_re_C_dot_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeqm_re_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeqm_re_C_dot_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_R_xeqm_re_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeqm_re_pC_dot_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_R_xeqm_re_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_R_xeqm_re_pC_dot_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* ---- rfield: replaces the F functions emitted by lib/perl/build_qla.pl:186-355 */
/* replaces QLA_F_I_veq_R_eq_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_R_eq_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_I_veq_R_eq_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_R_eq_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_I_veq_pR_eq_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_pR_eq_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_I_veq_pR_eq_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_pR_eq_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_I_xeq_R_eq_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_R_eq_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_I_xeq_R_eq_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_R_eq_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_I_xeq_pR_eq_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_pR_eq_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_I_xeq_pR_eq_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_pR_eq_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_I_veq_R_ge_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_R_ge_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_I_veq_R_ge_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_R_ge_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_I_veq_pR_ge_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_pR_ge_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_I_veq_pR_ge_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_pR_ge_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_I_xeq_R_ge_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_R_ge_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_I_xeq_R_ge_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_R_ge_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_I_xeq_pR_ge_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_pR_ge_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_I_xeq_pR_ge_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_pR_ge_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_I_veq_R_gt_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_R_gt_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_I_veq_R_gt_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_R_gt_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_I_veq_pR_gt_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_pR_gt_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_I_veq_pR_gt_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_pR_gt_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_I_xeq_R_gt_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_R_gt_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_I_xeq_R_gt_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_R_gt_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_I_xeq_pR_gt_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_pR_gt_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_I_xeq_pR_gt_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_pR_gt_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_I_veq_R_le_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_R_le_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_I_veq_R_le_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_R_le_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_I_veq_pR_le_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_pR_le_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_I_veq_pR_le_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_pR_le_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_I_xeq_R_le_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_R_le_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_I_xeq_R_le_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_R_le_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_I_xeq_pR_le_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_pR_le_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_I_xeq_pR_le_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_pR_le_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_I_veq_R_lt_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_R_lt_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_I_veq_R_lt_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_R_lt_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_I_veq_pR_lt_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_pR_lt_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_I_veq_pR_lt_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_pR_lt_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_I_xeq_R_lt_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_R_lt_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_I_xeq_R_lt_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_R_lt_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_I_xeq_pR_lt_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_pR_lt_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_I_xeq_pR_lt_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_pR_lt_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_I_veq_R_ne_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_R_ne_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_I_veq_R_ne_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_R_ne_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_I_veq_pR_ne_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_pR_ne_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_I_veq_pR_ne_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_pR_ne_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_I_xeq_R_ne_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_R_ne_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_I_xeq_R_ne_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_R_ne_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_I_xeq_pR_ne_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_pR_ne_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_I_xeq_pR_ne_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_pR_ne_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_I_veq_round_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_round_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_I_veq_round_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_round_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_I_xeq_round_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_round_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_I_xeq_round_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_round_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_I_veq_trunc_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_trunc_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_I_veq_trunc_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_veq_trunc_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_I_xeq_trunc_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_trunc_R(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_I_xeq_trunc_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_I_xeq_trunc_pR(QLA_Int *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* ---- sglobal: replaces the F functions emitted by lib/perl/build_qla.pl:186-355 */
/* replaces QLA_F_c_veq_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_c_veq_C_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_c_veq_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_c_veq_C_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_c_veq_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_c_veq_pC_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_c_veq_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_c_veq_pC_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_c_xeq_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_c_xeq_C_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_c_xeq_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_c_xeq_C_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_c_xeq_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_c_xeq_pC_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_c_xeq_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_c_xeq_pC_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_c_veq_Ca_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_c_veq_Ca_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_c_veq_Ca_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_c_veq_Ca_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_c_veq_pCa_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_c_veq_pCa_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_c_veq_pCa_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_c_veq_pCa_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_c_xeq_Ca_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_c_xeq_Ca_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_c_xeq_Ca_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_c_xeq_Ca_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_c_xeq_pCa_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_c_xeq_pCa_dot_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_c_xeq_pCa_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_c_xeq_pCa_dot_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_c_veq_sum_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_c_veq_sum_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_c_veq_sum_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_c_veq_sum_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_c_xeq_sum_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_c_xeq_sum_C(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_c_xeq_sum_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_c_xeq_sum_pC(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_r_veq_R_dot_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_veq_R_dot_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_r_veq_R_dot_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_veq_R_dot_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_r_veq_pR_dot_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_veq_pR_dot_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_r_veq_pR_dot_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_veq_pR_dot_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_r_xeq_R_dot_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_xeq_R_dot_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_r_xeq_R_dot_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_xeq_R_dot_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_r_xeq_pR_dot_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_xeq_pR_dot_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_r_xeq_pR_dot_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_xeq_pR_dot_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, QLA_F_Real *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_r_veq_I_dot_I (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_veq_I_dot_I(QLA_F_Real *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_r_veq_I_dot_pI (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_veq_I_dot_pI(QLA_F_Real *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_r_veq_pI_dot_I (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_veq_pI_dot_I(QLA_F_Real *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_r_veq_pI_dot_pI (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_veq_pI_dot_pI(QLA_F_Real *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_r_xeq_I_dot_I (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_xeq_I_dot_I(QLA_F_Real *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_r_xeq_I_dot_pI (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_xeq_I_dot_pI(QLA_F_Real *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_r_xeq_pI_dot_I (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_xeq_pI_dot_I(QLA_F_Real *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_r_xeq_pI_dot_pI (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_xeq_pI_dot_pI(QLA_F_Real *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_r_veq_norm2_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_veq_norm2_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_r_veq_norm2_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_veq_norm2_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_r_xeq_norm2_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_xeq_norm2_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_r_xeq_norm2_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_xeq_norm2_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_r_veq_norm2_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_veq_norm2_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_r_veq_norm2_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_veq_norm2_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_r_xeq_norm2_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_xeq_norm2_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_r_xeq_norm2_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_xeq_norm2_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_r_veq_norm2_I (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_veq_norm2_I(QLA_F_Real *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_r_veq_norm2_pI (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_veq_norm2_pI(QLA_F_Real *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_r_xeq_norm2_I (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_xeq_norm2_I(QLA_F_Real *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_r_xeq_norm2_pI (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_xeq_norm2_pI(QLA_F_Real *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_r_veq_re_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_veq_re_C_dot_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_r_veq_re_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_veq_re_C_dot_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_r_veq_re_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_veq_re_pC_dot_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int n);
/* replaces QLA_F_r_veq_re_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_veq_re_pC_dot_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_F_r_xeq_re_C_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_xeq_re_C_dot_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_r_xeq_re_C_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_xeq_re_C_dot_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_r_xeq_re_pC_dot_C (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_xeq_re_pC_dot_C(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_F_r_xeq_re_pC_dot_pC (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_xeq_re_pC_dot_pC(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Complex *QLA_B200_RESTRICT * a, QLA_F_Complex *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_F_r_veq_sum_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_veq_sum_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_r_veq_sum_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_veq_sum_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_r_xeq_sum_R (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_xeq_sum_R(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_r_xeq_sum_pR (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_xeq_sum_pR(QLA_F_Real *QLA_B200_RESTRICT r, QLA_F_Real *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_r_veq_sum_I (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_veq_sum_I(QLA_F_Real *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_r_veq_sum_pI (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_veq_sum_pI(QLA_F_Real *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_r_xeq_sum_I (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_xeq_sum_I(QLA_F_Real *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_r_xeq_sum_pI (lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath) */
void QLA_F_r_xeq_sum_pI(QLA_F_Real *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, int * index, int n);
/* ---- random: replaces the F functions emitted by lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills */
/* replaces QLA_F_R_veq_random_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_F_R_veq_random_S(QLA_F_Real *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_gaussian_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_F_R_veq_gaussian_S(QLA_F_Real *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_C_veq_gaussian_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_F_C_veq_gaussian_S(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT a, int n);
/* replaces QLA_F_R_veq_random_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_F_R_veq_random_pS(QLA_F_Real *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_veq_gaussian_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_F_R_veq_gaussian_pS(QLA_F_Real *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_C_veq_gaussian_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_F_C_veq_gaussian_pS(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_F_R_xeq_random_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_F_R_xeq_random_S(QLA_F_Real *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_gaussian_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_F_R_xeq_gaussian_S(QLA_F_Real *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_C_xeq_gaussian_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_F_C_xeq_gaussian_S(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_F_R_xeq_random_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_F_R_xeq_random_pS(QLA_F_Real *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_R_xeq_gaussian_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_F_R_xeq_gaussian_pS(QLA_F_Real *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_F_C_xeq_gaussian_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_F_C_xeq_gaussian_pS(QLA_F_Complex *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT * a, int * index, int n);

#ifdef __cplusplus
}
#endif
#endif
