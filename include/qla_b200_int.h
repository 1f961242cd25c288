/*
 * qla_b200_int.h -- GENERATED by qla_b200/gen/gen_qla.py; do not edit.
 *
 * QLA I level-1 entry points implemented by libqla_b200.so (sm_100a).
 * Each declaration replaces the reference function of the same name, whose
 * C loop the reference generator emits from the cited section.  Array
 * arguments are device pointers; see qla_b200_runtime.h for scalars,
 * reduction outputs, streams and errors.
 */
#ifndef QLA_B200_I_H
#define QLA_B200_I_H
#include "qla_b200_types.h"

#ifdef __cplusplus
#define QLA_B200_RESTRICT __restrict__
extern "C" {
#else
#define QLA_B200_RESTRICT restrict
#endif

/* ---- int: replaces the I functions emitted by lib/perl/build_qla.pl:1932-2082 (integer fields) */
/* replaces QLA_I_veq_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int n);
/* replaces QLA_I_veq_I_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_I_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_i_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_i_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_I_veq_pI_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_pI_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_i_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_i_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_i (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_i(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int n);
/* replaces QLA_I_vpeq_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_vpeq_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int n);
/* replaces QLA_I_vpeq_I_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_vpeq_I_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_vpeq_I_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_vpeq_I_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_vpeq_i_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_vpeq_i_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_vpeq_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_vpeq_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_I_vpeq_pI_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_vpeq_pI_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_vpeq_pI_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_vpeq_pI_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_vpeq_i_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_vpeq_i_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_vpeq_i (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_vpeq_i(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int n);
/* replaces QLA_I_vmeq_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_vmeq_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int n);
/* replaces QLA_I_vmeq_I_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_vmeq_I_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_vmeq_I_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_vmeq_I_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_vmeq_i_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_vmeq_i_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_vmeq_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_vmeq_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_I_vmeq_pI_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_vmeq_pI_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_vmeq_pI_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_vmeq_pI_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_vmeq_i_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_vmeq_i_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_vmeq_i (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_vmeq_i(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int n);
/* replaces QLA_I_veqm_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veqm_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int n);
/* replaces QLA_I_veqm_I_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veqm_I_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veqm_I_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veqm_I_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veqm_i_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veqm_i_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veqm_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veqm_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_I_veqm_pI_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veqm_pI_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veqm_pI_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veqm_pI_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veqm_i_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veqm_i_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veqm_i (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veqm_i(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int n);
/* replaces QLA_I_veq_I_and_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_and_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_I_and_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_and_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_pI_and_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_and_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_pI_and_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_and_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_I_divide_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_divide_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_I_divide_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_divide_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_pI_divide_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_divide_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_pI_divide_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_divide_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_I_eq_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_eq_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_I_eq_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_eq_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_pI_eq_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_eq_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_pI_eq_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_eq_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_I_ge_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_ge_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_I_ge_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_ge_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_pI_ge_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_ge_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_pI_ge_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_ge_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_I_gt_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_gt_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_I_gt_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_gt_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_pI_gt_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_gt_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_pI_gt_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_gt_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_I_le_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_le_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_I_le_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_le_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_pI_le_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_le_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_pI_le_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_le_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_I_lshift_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_lshift_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_I_lshift_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_lshift_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_pI_lshift_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_lshift_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_pI_lshift_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_lshift_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_I_lt_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_lt_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_I_lt_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_lt_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_pI_lt_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_lt_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_pI_lt_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_lt_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_I_mask_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_mask_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_I_mask_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_mask_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_pI_mask_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_mask_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_pI_mask_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_mask_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_I_max_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_max_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_I_max_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_max_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_pI_max_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_max_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_pI_max_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_max_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_I_min_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_min_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_I_min_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_min_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_pI_min_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_min_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_pI_min_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_min_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_I_minus_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_minus_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_I_minus_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_minus_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_pI_minus_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_minus_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_pI_minus_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_minus_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_I_mod_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_mod_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_I_mod_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_mod_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_pI_mod_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_mod_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_pI_mod_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_mod_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_I_ne_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_ne_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_I_ne_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_ne_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_pI_ne_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_ne_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_pI_ne_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_ne_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_I_or_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_or_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_I_or_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_or_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_pI_or_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_or_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_pI_or_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_or_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_I_plus_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_plus_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_I_plus_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_plus_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_pI_plus_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_plus_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_pI_plus_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_plus_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_I_rshift_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_rshift_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_I_rshift_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_rshift_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_pI_rshift_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_rshift_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_pI_rshift_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_rshift_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_I_xor_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_xor_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_I_xor_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_I_xor_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_pI_xor_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_xor_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_I_veq_pI_xor_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_pI_xor_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_I_veq_i_times_I_plus_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_i_times_I_plus_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, QLA_Int *QLA_B200_RESTRICT c, int n);
/* replaces QLA_I_veq_i_times_I_plus_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_i_times_I_plus_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, QLA_Int *QLA_B200_RESTRICT * c, int n);
/* replaces QLA_I_veq_i_times_I_minus_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_i_times_I_minus_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, QLA_Int *QLA_B200_RESTRICT c, int n);
/* replaces QLA_I_veq_i_times_I_minus_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_i_times_I_minus_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, QLA_Int *QLA_B200_RESTRICT * c, int n);
/* replaces QLA_I_veq_not_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_not_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int n);
/* replaces QLA_I_veq_i_times_pI_plus_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_i_times_pI_plus_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, QLA_Int *QLA_B200_RESTRICT c, int n);
/* replaces QLA_I_veq_i_times_pI_plus_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_i_times_pI_plus_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, QLA_Int *QLA_B200_RESTRICT * c, int n);
/* replaces QLA_I_veq_i_times_pI_minus_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_i_times_pI_minus_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, QLA_Int *QLA_B200_RESTRICT c, int n);
/* replaces QLA_I_veq_i_times_pI_minus_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_i_times_pI_minus_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, QLA_Int *QLA_B200_RESTRICT * c, int n);
/* replaces QLA_I_veq_not_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_not_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_I_veq_zero (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_veq_zero(QLA_Int *QLA_B200_RESTRICT r, int n);
/* replaces QLA_I_xeq_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_I_xeq_I_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_I_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_i_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_i_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_I_xeq_pI_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_pI_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_i_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_i_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_i (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_i(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_I_xpeq_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xpeq_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_I_xpeq_I_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xpeq_I_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xpeq_I_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xpeq_I_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xpeq_i_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xpeq_i_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xpeq_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xpeq_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_I_xpeq_pI_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xpeq_pI_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xpeq_pI_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xpeq_pI_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xpeq_i_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xpeq_i_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xpeq_i (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xpeq_i(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_I_xmeq_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xmeq_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_I_xmeq_I_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xmeq_I_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xmeq_I_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xmeq_I_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xmeq_i_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xmeq_i_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xmeq_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xmeq_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_I_xmeq_pI_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xmeq_pI_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xmeq_pI_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xmeq_pI_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xmeq_i_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xmeq_i_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xmeq_i (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xmeq_i(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_I_xeqm_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeqm_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_I_xeqm_I_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeqm_I_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeqm_I_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeqm_I_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeqm_i_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeqm_i_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeqm_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeqm_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_I_xeqm_pI_times_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeqm_pI_times_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeqm_pI_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeqm_pI_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeqm_i_times_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeqm_i_times_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeqm_i (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeqm_i(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_I_xeq_I_and_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_and_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_I_and_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_and_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_pI_and_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_and_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_pI_and_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_and_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_I_divide_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_divide_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_I_divide_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_divide_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_pI_divide_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_divide_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_pI_divide_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_divide_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_I_eq_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_eq_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_I_eq_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_eq_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_pI_eq_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_eq_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_pI_eq_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_eq_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_I_ge_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_ge_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_I_ge_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_ge_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_pI_ge_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_ge_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_pI_ge_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_ge_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_I_gt_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_gt_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_I_gt_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_gt_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_pI_gt_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_gt_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_pI_gt_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_gt_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_I_le_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_le_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_I_le_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_le_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_pI_le_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_le_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_pI_le_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_le_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_I_lshift_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_lshift_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_I_lshift_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_lshift_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_pI_lshift_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_lshift_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_pI_lshift_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_lshift_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_I_lt_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_lt_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_I_lt_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_lt_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_pI_lt_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_lt_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_pI_lt_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_lt_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_I_mask_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_mask_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_I_mask_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_mask_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_pI_mask_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_mask_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_pI_mask_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_mask_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_I_max_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_max_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_I_max_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_max_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_pI_max_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_max_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_pI_max_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_max_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_I_min_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_min_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_I_min_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_min_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_pI_min_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_min_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_pI_min_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_min_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_I_minus_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_minus_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_I_minus_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_minus_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_pI_minus_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_minus_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_pI_minus_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_minus_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_I_mod_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_mod_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_I_mod_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_mod_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_pI_mod_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_mod_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_pI_mod_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_mod_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_I_ne_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_ne_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_I_ne_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_ne_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_pI_ne_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_ne_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_pI_ne_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_ne_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_I_or_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_or_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_I_or_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_or_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_pI_or_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_or_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_pI_or_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_or_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_I_plus_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_plus_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_I_plus_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_plus_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_pI_plus_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_plus_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_pI_plus_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_plus_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_I_rshift_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_rshift_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_I_rshift_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_rshift_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_pI_rshift_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_rshift_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_pI_rshift_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_rshift_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_I_xor_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_xor_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_I_xor_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_I_xor_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_pI_xor_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_xor_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_I_xeq_pI_xor_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_pI_xor_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_I_xeq_i_times_I_plus_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_i_times_I_plus_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, QLA_Int *QLA_B200_RESTRICT c, int * index, int n);
/* replaces QLA_I_xeq_i_times_I_plus_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_i_times_I_plus_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, QLA_Int *QLA_B200_RESTRICT * c, int * index, int n);
/* replaces QLA_I_xeq_i_times_I_minus_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_i_times_I_minus_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, QLA_Int *QLA_B200_RESTRICT c, int * index, int n);
/* replaces QLA_I_xeq_i_times_I_minus_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_i_times_I_minus_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, QLA_Int *QLA_B200_RESTRICT * c, int * index, int n);
/* replaces QLA_I_xeq_not_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_not_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_I_xeq_i_times_pI_plus_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_i_times_pI_plus_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, QLA_Int *QLA_B200_RESTRICT c, int * index, int n);
/* replaces QLA_I_xeq_i_times_pI_plus_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_i_times_pI_plus_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, QLA_Int *QLA_B200_RESTRICT * c, int * index, int n);
/* replaces QLA_I_xeq_i_times_pI_minus_I (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_i_times_pI_minus_I(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, QLA_Int *QLA_B200_RESTRICT c, int * index, int n);
/* replaces QLA_I_xeq_i_times_pI_minus_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_i_times_pI_minus_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, QLA_Int *QLA_B200_RESTRICT * c, int * index, int n);
/* replaces QLA_I_xeq_not_pI (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_not_pI(QLA_Int *QLA_B200_RESTRICT r, QLA_Int *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_I_xeq_zero (lib/perl/build_qla.pl:1932-2082 (integer fields)) */
void QLA_I_xeq_zero(QLA_Int *QLA_B200_RESTRICT r, int * index, int n);
/* ---- random: replaces the I functions emitted by lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills */
/* replaces QLA_S_veq_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_S_veq_S(QLA_RandomState *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT a, int n);
/* replaces QLA_S_veq_S_mask_I (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_S_veq_S_mask_I(QLA_RandomState *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_S_veq_S_mask_pI (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_S_veq_S_mask_pI(QLA_RandomState *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_S_veq_seed_i_I (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_S_veq_seed_i_I(QLA_RandomState *QLA_B200_RESTRICT r, int seed, QLA_Int *QLA_B200_RESTRICT a, int n);
/* replaces QLA_S_veq_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_S_veq_pS(QLA_RandomState *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_S_veq_pS_mask_I (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_S_veq_pS_mask_I(QLA_RandomState *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_S_veq_pS_mask_pI (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_S_veq_pS_mask_pI(QLA_RandomState *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_S_veq_seed_i_pI (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_S_veq_seed_i_pI(QLA_RandomState *QLA_B200_RESTRICT r, int seed, QLA_Int *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_S_xeq_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_S_xeq_S(QLA_RandomState *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_S_xeq_S_mask_I (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_S_xeq_S_mask_I(QLA_RandomState *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_S_xeq_S_mask_pI (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_S_xeq_S_mask_pI(QLA_RandomState *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_S_xeq_seed_i_I (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_S_xeq_seed_i_I(QLA_RandomState *QLA_B200_RESTRICT r, int seed, QLA_Int *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_S_xeq_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_S_xeq_pS(QLA_RandomState *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_S_xeq_pS_mask_I (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_S_xeq_pS_mask_I(QLA_RandomState *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_S_xeq_pS_mask_pI (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_S_xeq_pS_mask_pI(QLA_RandomState *QLA_B200_RESTRICT r, QLA_RandomState *QLA_B200_RESTRICT * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_S_xeq_seed_i_pI (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_S_xeq_seed_i_pI(QLA_RandomState *QLA_B200_RESTRICT r, int seed, QLA_Int *QLA_B200_RESTRICT * a, int * index, int n);

#ifdef __cplusplus
}
#endif
#endif
