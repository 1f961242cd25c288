/*
 * qla_b200_fn.h -- GENERATED by qla_b200/gen/gen_qla.py; do not edit.
 *
 * QLA FN level-1 entry points implemented by libqla_b200.so (sm_100a).
 * Each declaration replaces the reference function of the same name, whose
 * C loop the reference generator emits from the cited section.  Array
 * arguments are device pointers; see qla_b200_runtime.h for scalars,
 * reduction outputs, streams and errors.
 */
#ifndef QLA_B200_FN_H
#define QLA_B200_FN_H
#include "qla_b200_types.h"

#ifdef __cplusplus
#define QLA_B200_RESTRICT __restrict__
extern "C" {
#else
#define QLA_B200_RESTRICT restrict
#endif

/* ---- lmult: replaces the FN functions emitted by lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix) */
/* replaces QLA_FN_V_veq_M_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_veq_M_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veq_M_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_veq_M_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veq_Ma_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_veq_Ma_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veq_Ma_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_veq_Ma_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veq_pM_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_veq_pM_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veq_pM_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_veq_pM_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veq_pMa_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_veq_pMa_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veq_pMa_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_veq_pMa_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_vpeq_M_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_vpeq_M_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_vpeq_M_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_vpeq_M_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_vpeq_Ma_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_vpeq_Ma_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_vpeq_Ma_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_vpeq_Ma_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_vpeq_pM_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_vpeq_pM_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_vpeq_pM_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_vpeq_pM_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_vpeq_pMa_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_vpeq_pMa_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_vpeq_pMa_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_vpeq_pMa_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_vmeq_M_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_vmeq_M_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_vmeq_M_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_vmeq_M_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_vmeq_Ma_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_vmeq_Ma_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_vmeq_Ma_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_vmeq_Ma_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_vmeq_pM_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_vmeq_pM_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_vmeq_pM_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_vmeq_pM_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_vmeq_pMa_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_vmeq_pMa_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_vmeq_pMa_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_vmeq_pMa_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veqm_M_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_veqm_M_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veqm_M_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_veqm_M_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veqm_Ma_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_veqm_Ma_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veqm_Ma_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_veqm_Ma_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veqm_pM_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_veqm_pM_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veqm_pM_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_veqm_pM_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veqm_pMa_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_veqm_pMa_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veqm_pMa_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_veqm_pMa_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_xeq_M_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xeq_M_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_M_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xeq_M_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_Ma_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xeq_Ma_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_Ma_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xeq_Ma_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_pM_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xeq_pM_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_pM_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xeq_pM_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_pMa_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xeq_pMa_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_pMa_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xeq_pMa_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xpeq_M_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xpeq_M_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xpeq_M_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xpeq_M_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xpeq_Ma_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xpeq_Ma_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xpeq_Ma_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xpeq_Ma_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xpeq_pM_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xpeq_pM_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xpeq_pM_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xpeq_pM_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xpeq_pMa_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xpeq_pMa_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xpeq_pMa_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xpeq_pMa_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xmeq_M_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xmeq_M_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xmeq_M_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xmeq_M_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xmeq_Ma_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xmeq_Ma_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xmeq_Ma_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xmeq_Ma_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xmeq_pM_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xmeq_pM_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xmeq_pM_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xmeq_pM_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xmeq_pMa_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xmeq_pMa_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xmeq_pMa_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xmeq_pMa_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeqm_M_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xeqm_M_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeqm_M_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xeqm_M_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeqm_Ma_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xeqm_Ma_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeqm_Ma_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xeqm_Ma_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeqm_pM_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xeqm_pM_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeqm_pM_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xeqm_pM_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeqm_pMa_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xeqm_pMa_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeqm_pMa_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_V_xeqm_pMa_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_eq_M_times_xV (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_V_eq_M_times_xV(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_V_eq_Ma_times_xV (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_V_eq_Ma_times_xV(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_V_peq_M_times_xV (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_V_peq_M_times_xV(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_V_peq_Ma_times_xV (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_V_peq_Ma_times_xV(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_V_meq_M_times_xV (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_V_meq_M_times_xV(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_V_meq_Ma_times_xV (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_V_meq_Ma_times_xV(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_V_eqm_M_times_xV (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_V_eqm_M_times_xV(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_V_eqm_Ma_times_xV (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_V_eqm_Ma_times_xV(int nc, void * r, void * a, void * b, int * jb, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_V_veq_r_times_V (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_V_veq_r_times_V(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_V_veq_V (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_V_veq_V(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_V_veq_r_times_pV (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_V_veq_r_times_pV(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_V_veq_pV (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_V_veq_pV(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_V_vpeq_r_times_V (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_V_vpeq_r_times_V(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_V_vpeq_V (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_V_vpeq_V(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_V_vpeq_r_times_pV (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_V_vpeq_r_times_pV(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_V_vpeq_pV (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_V_vpeq_pV(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_V_vmeq_r_times_V (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_V_vmeq_r_times_V(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_V_vmeq_V (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_V_vmeq_V(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_V_vmeq_r_times_pV (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_V_vmeq_r_times_pV(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_V_vmeq_pV (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_V_vmeq_pV(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_V_veqm_r_times_V (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_V_veqm_r_times_V(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_V_veqm_V (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_V_veqm_V(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_V_veqm_r_times_pV (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_V_veqm_r_times_pV(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_V_veqm_pV (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_V_veqm_pV(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_V_xeq_r_times_V (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_V_xeq_r_times_V(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_V_xeq_V (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_V_xeq_V(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_V_xeq_r_times_pV (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_V_xeq_r_times_pV(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_V_xeq_pV (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_V_xeq_pV(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_V_xpeq_r_times_V (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_V_xpeq_r_times_V(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_V_xpeq_V (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_V_xpeq_V(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_V_xpeq_r_times_pV (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_V_xpeq_r_times_pV(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_V_xpeq_pV (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_V_xpeq_pV(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_V_xmeq_r_times_V (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_V_xmeq_r_times_V(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_V_xmeq_V (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_V_xmeq_V(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_V_xmeq_r_times_pV (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_V_xmeq_r_times_pV(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_V_xmeq_pV (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_V_xmeq_pV(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_V_xeqm_r_times_V (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_V_xeqm_r_times_V(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_V_xeqm_V (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_V_xeqm_V(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_V_xeqm_r_times_pV (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_V_xeqm_r_times_pV(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_V_xeqm_pV (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_V_xeqm_pV(int nc, void * r, void * a, int * index, int n);
/* ---- norm2: replaces the FN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_FN_r_veq_norm2_V (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_FN_r_veq_norm2_V(int nc, QLA_F_Real * r, void * a, int n);
/* replaces QLA_FN_r_veq_norm2_pV (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_FN_r_veq_norm2_pV(int nc, QLA_F_Real * r, void * a, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_veq_V_dot_V (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_veq_V_dot_V(int nc, QLA_F_Complex * r, void * a, void * b, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_veq_re_V_dot_V (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_veq_re_V_dot_V(int nc, QLA_F_Real * r, void * a, void * b, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_veq_V_dot_pV (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_veq_V_dot_pV(int nc, QLA_F_Complex * r, void * a, void * b, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_veq_re_V_dot_pV (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_veq_re_V_dot_pV(int nc, QLA_F_Real * r, void * a, void * b, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_veq_pV_dot_V (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_veq_pV_dot_V(int nc, QLA_F_Complex * r, void * a, void * b, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_veq_re_pV_dot_V (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_veq_re_pV_dot_V(int nc, QLA_F_Real * r, void * a, void * b, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_veq_pV_dot_pV (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_veq_pV_dot_pV(int nc, QLA_F_Complex * r, void * a, void * b, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_veq_re_pV_dot_pV (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_veq_re_pV_dot_pV(int nc, QLA_F_Real * r, void * a, void * b, int n);
/* ---- norm2: replaces the FN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_FN_r_xeq_norm2_V (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_FN_r_xeq_norm2_V(int nc, QLA_F_Real * r, void * a, int * index, int n);
/* replaces QLA_FN_r_xeq_norm2_pV (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_FN_r_xeq_norm2_pV(int nc, QLA_F_Real * r, void * a, int * index, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_xeq_V_dot_V (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_xeq_V_dot_V(int nc, QLA_F_Complex * r, void * a, void * b, int * index, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_xeq_re_V_dot_V (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_xeq_re_V_dot_V(int nc, QLA_F_Real * r, void * a, void * b, int * index, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_xeq_V_dot_pV (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_xeq_V_dot_pV(int nc, QLA_F_Complex * r, void * a, void * b, int * index, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_xeq_re_V_dot_pV (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_xeq_re_V_dot_pV(int nc, QLA_F_Real * r, void * a, void * b, int * index, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_xeq_pV_dot_V (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_xeq_pV_dot_V(int nc, QLA_F_Complex * r, void * a, void * b, int * index, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_xeq_re_pV_dot_V (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_xeq_re_pV_dot_V(int nc, QLA_F_Real * r, void * a, void * b, int * index, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_xeq_pV_dot_pV (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_xeq_pV_dot_pV(int nc, QLA_F_Complex * r, void * a, void * b, int * index, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_xeq_re_pV_dot_pV (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_xeq_re_pV_dot_pV(int nc, QLA_F_Real * r, void * a, void * b, int * index, int n);
/* ---- lmult: replaces the FN functions emitted by lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix) */
/* replaces QLA_FN_H_veq_M_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_veq_M_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_veq_M_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_veq_M_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_veq_Ma_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_veq_Ma_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_veq_Ma_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_veq_Ma_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_veq_pM_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_veq_pM_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_veq_pM_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_veq_pM_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_veq_pMa_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_veq_pMa_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_veq_pMa_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_veq_pMa_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_vpeq_M_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_vpeq_M_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_vpeq_M_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_vpeq_M_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_vpeq_Ma_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_vpeq_Ma_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_vpeq_Ma_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_vpeq_Ma_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_vpeq_pM_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_vpeq_pM_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_vpeq_pM_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_vpeq_pM_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_vpeq_pMa_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_vpeq_pMa_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_vpeq_pMa_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_vpeq_pMa_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_vmeq_M_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_vmeq_M_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_vmeq_M_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_vmeq_M_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_vmeq_Ma_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_vmeq_Ma_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_vmeq_Ma_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_vmeq_Ma_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_vmeq_pM_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_vmeq_pM_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_vmeq_pM_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_vmeq_pM_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_vmeq_pMa_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_vmeq_pMa_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_vmeq_pMa_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_vmeq_pMa_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_veqm_M_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_veqm_M_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_veqm_M_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_veqm_M_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_veqm_Ma_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_veqm_Ma_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_veqm_Ma_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_veqm_Ma_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_veqm_pM_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_veqm_pM_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_veqm_pM_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_veqm_pM_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_veqm_pMa_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_veqm_pMa_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_veqm_pMa_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_veqm_pMa_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_xeq_M_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xeq_M_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_M_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xeq_M_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_Ma_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xeq_Ma_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_Ma_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xeq_Ma_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_pM_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xeq_pM_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_pM_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xeq_pM_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_pMa_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xeq_pMa_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_pMa_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xeq_pMa_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xpeq_M_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xpeq_M_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xpeq_M_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xpeq_M_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xpeq_Ma_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xpeq_Ma_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xpeq_Ma_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xpeq_Ma_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xpeq_pM_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xpeq_pM_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xpeq_pM_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xpeq_pM_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xpeq_pMa_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xpeq_pMa_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xpeq_pMa_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xpeq_pMa_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xmeq_M_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xmeq_M_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xmeq_M_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xmeq_M_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xmeq_Ma_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xmeq_Ma_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xmeq_Ma_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xmeq_Ma_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xmeq_pM_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xmeq_pM_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xmeq_pM_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xmeq_pM_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xmeq_pMa_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xmeq_pMa_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xmeq_pMa_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xmeq_pMa_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeqm_M_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xeqm_M_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeqm_M_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xeqm_M_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeqm_Ma_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xeqm_Ma_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeqm_Ma_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xeqm_Ma_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeqm_pM_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xeqm_pM_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeqm_pM_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xeqm_pM_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeqm_pMa_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xeqm_pMa_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeqm_pMa_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_H_xeqm_pMa_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_eq_M_times_xH (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_H_eq_M_times_xH(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_H_eq_Ma_times_xH (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_H_eq_Ma_times_xH(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_H_peq_M_times_xH (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_H_peq_M_times_xH(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_H_peq_Ma_times_xH (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_H_peq_Ma_times_xH(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_H_meq_M_times_xH (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_H_meq_M_times_xH(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_H_meq_Ma_times_xH (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_H_meq_Ma_times_xH(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_H_eqm_M_times_xH (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_H_eqm_M_times_xH(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_H_eqm_Ma_times_xH (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_H_eqm_Ma_times_xH(int nc, void * r, void * a, void * b, int * jb, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_H_veq_r_times_H (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_H_veq_r_times_H(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_H_veq_H (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_H_veq_H(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_H_veq_r_times_pH (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_H_veq_r_times_pH(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_H_veq_pH (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_H_veq_pH(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_H_vpeq_r_times_H (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_H_vpeq_r_times_H(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_H_vpeq_H (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_H_vpeq_H(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_H_vpeq_r_times_pH (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_H_vpeq_r_times_pH(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_H_vpeq_pH (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_H_vpeq_pH(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_H_vmeq_r_times_H (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_H_vmeq_r_times_H(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_H_vmeq_H (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_H_vmeq_H(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_H_vmeq_r_times_pH (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_H_vmeq_r_times_pH(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_H_vmeq_pH (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_H_vmeq_pH(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_H_veqm_r_times_H (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_H_veqm_r_times_H(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_H_veqm_H (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_H_veqm_H(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_H_veqm_r_times_pH (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_H_veqm_r_times_pH(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_H_veqm_pH (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_H_veqm_pH(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_H_xeq_r_times_H (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_H_xeq_r_times_H(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_H_xeq_H (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_H_xeq_H(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_H_xeq_r_times_pH (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_H_xeq_r_times_pH(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_H_xeq_pH (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_H_xeq_pH(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_H_xpeq_r_times_H (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_H_xpeq_r_times_H(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_H_xpeq_H (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_H_xpeq_H(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_H_xpeq_r_times_pH (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_H_xpeq_r_times_pH(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_H_xpeq_pH (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_H_xpeq_pH(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_H_xmeq_r_times_H (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_H_xmeq_r_times_H(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_H_xmeq_H (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_H_xmeq_H(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_H_xmeq_r_times_pH (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_H_xmeq_r_times_pH(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_H_xmeq_pH (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_H_xmeq_pH(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_H_xeqm_r_times_H (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_H_xeqm_r_times_H(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_H_xeqm_H (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_H_xeqm_H(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_H_xeqm_r_times_pH (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_H_xeqm_r_times_pH(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_H_xeqm_pH (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_H_xeqm_pH(int nc, void * r, void * a, int * index, int n);
/* ---- norm2: replaces the FN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_FN_r_veq_norm2_H (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_FN_r_veq_norm2_H(int nc, QLA_F_Real * r, void * a, int n);
/* replaces QLA_FN_r_veq_norm2_pH (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_FN_r_veq_norm2_pH(int nc, QLA_F_Real * r, void * a, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_veq_H_dot_H (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_veq_H_dot_H(int nc, QLA_F_Complex * r, void * a, void * b, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_veq_re_H_dot_H (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_veq_re_H_dot_H(int nc, QLA_F_Real * r, void * a, void * b, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_veq_H_dot_pH (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_veq_H_dot_pH(int nc, QLA_F_Complex * r, void * a, void * b, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_veq_re_H_dot_pH (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_veq_re_H_dot_pH(int nc, QLA_F_Real * r, void * a, void * b, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_veq_pH_dot_H (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_veq_pH_dot_H(int nc, QLA_F_Complex * r, void * a, void * b, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_veq_re_pH_dot_H (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_veq_re_pH_dot_H(int nc, QLA_F_Real * r, void * a, void * b, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_veq_pH_dot_pH (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_veq_pH_dot_pH(int nc, QLA_F_Complex * r, void * a, void * b, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_veq_re_pH_dot_pH (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_veq_re_pH_dot_pH(int nc, QLA_F_Real * r, void * a, void * b, int n);
/* ---- norm2: replaces the FN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_FN_r_xeq_norm2_H (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_FN_r_xeq_norm2_H(int nc, QLA_F_Real * r, void * a, int * index, int n);
/* replaces QLA_FN_r_xeq_norm2_pH (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_FN_r_xeq_norm2_pH(int nc, QLA_F_Real * r, void * a, int * index, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_xeq_H_dot_H (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_xeq_H_dot_H(int nc, QLA_F_Complex * r, void * a, void * b, int * index, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_xeq_re_H_dot_H (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_xeq_re_H_dot_H(int nc, QLA_F_Real * r, void * a, void * b, int * index, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_xeq_H_dot_pH (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_xeq_H_dot_pH(int nc, QLA_F_Complex * r, void * a, void * b, int * index, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_xeq_re_H_dot_pH (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_xeq_re_H_dot_pH(int nc, QLA_F_Real * r, void * a, void * b, int * index, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_xeq_pH_dot_H (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_xeq_pH_dot_H(int nc, QLA_F_Complex * r, void * a, void * b, int * index, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_xeq_re_pH_dot_H (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_xeq_re_pH_dot_H(int nc, QLA_F_Real * r, void * a, void * b, int * index, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_xeq_pH_dot_pH (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_xeq_pH_dot_pH(int nc, QLA_F_Complex * r, void * a, void * b, int * index, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_xeq_re_pH_dot_pH (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_xeq_re_pH_dot_pH(int nc, QLA_F_Real * r, void * a, void * b, int * index, int n);
/* ---- lmult: replaces the FN functions emitted by lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix) */
/* replaces QLA_FN_D_veq_M_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_veq_M_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_veq_M_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_veq_M_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_veq_Ma_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_veq_Ma_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_veq_Ma_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_veq_Ma_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_veq_pM_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_veq_pM_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_veq_pM_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_veq_pM_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_veq_pMa_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_veq_pMa_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_veq_pMa_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_veq_pMa_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_vpeq_M_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_vpeq_M_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_vpeq_M_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_vpeq_M_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_vpeq_Ma_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_vpeq_Ma_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_vpeq_Ma_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_vpeq_Ma_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_vpeq_pM_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_vpeq_pM_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_vpeq_pM_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_vpeq_pM_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_vpeq_pMa_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_vpeq_pMa_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_vpeq_pMa_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_vpeq_pMa_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_vmeq_M_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_vmeq_M_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_vmeq_M_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_vmeq_M_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_vmeq_Ma_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_vmeq_Ma_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_vmeq_Ma_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_vmeq_Ma_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_vmeq_pM_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_vmeq_pM_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_vmeq_pM_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_vmeq_pM_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_vmeq_pMa_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_vmeq_pMa_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_vmeq_pMa_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_vmeq_pMa_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_veqm_M_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_veqm_M_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_veqm_M_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_veqm_M_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_veqm_Ma_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_veqm_Ma_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_veqm_Ma_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_veqm_Ma_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_veqm_pM_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_veqm_pM_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_veqm_pM_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_veqm_pM_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_veqm_pMa_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_veqm_pMa_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_veqm_pMa_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_veqm_pMa_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_xeq_M_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xeq_M_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_M_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xeq_M_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_Ma_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xeq_Ma_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_Ma_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xeq_Ma_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_pM_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xeq_pM_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_pM_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xeq_pM_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_pMa_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xeq_pMa_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_pMa_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xeq_pMa_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xpeq_M_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xpeq_M_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xpeq_M_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xpeq_M_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xpeq_Ma_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xpeq_Ma_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xpeq_Ma_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xpeq_Ma_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xpeq_pM_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xpeq_pM_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xpeq_pM_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xpeq_pM_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xpeq_pMa_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xpeq_pMa_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xpeq_pMa_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xpeq_pMa_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xmeq_M_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xmeq_M_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xmeq_M_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xmeq_M_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xmeq_Ma_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xmeq_Ma_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xmeq_Ma_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xmeq_Ma_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xmeq_pM_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xmeq_pM_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xmeq_pM_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xmeq_pM_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xmeq_pMa_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xmeq_pMa_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xmeq_pMa_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xmeq_pMa_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeqm_M_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xeqm_M_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeqm_M_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xeqm_M_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeqm_Ma_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xeqm_Ma_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeqm_Ma_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xeqm_Ma_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeqm_pM_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xeqm_pM_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeqm_pM_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xeqm_pM_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeqm_pMa_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xeqm_pMa_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeqm_pMa_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_D_xeqm_pMa_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_eq_M_times_xD (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_D_eq_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_D_eq_Ma_times_xD (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_D_eq_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_D_peq_M_times_xD (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_D_peq_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_D_peq_Ma_times_xD (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_D_peq_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_D_meq_M_times_xD (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_D_meq_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_D_meq_Ma_times_xD (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_D_meq_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_D_eqm_M_times_xD (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_D_eqm_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_D_eqm_Ma_times_xD (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_D_eqm_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_D_veq_r_times_D (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_D_veq_r_times_D(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_D_veq_D (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_D_veq_D(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_D_veq_r_times_pD (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_D_veq_r_times_pD(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_D_veq_pD (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_D_veq_pD(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_D_vpeq_r_times_D (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_D_vpeq_r_times_D(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_D_vpeq_D (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_D_vpeq_D(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_D_vpeq_r_times_pD (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_D_vpeq_r_times_pD(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_D_vpeq_pD (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_D_vpeq_pD(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_D_vmeq_r_times_D (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_D_vmeq_r_times_D(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_D_vmeq_D (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_D_vmeq_D(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_D_vmeq_r_times_pD (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_D_vmeq_r_times_pD(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_D_vmeq_pD (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_D_vmeq_pD(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_D_veqm_r_times_D (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_D_veqm_r_times_D(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_D_veqm_D (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_D_veqm_D(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_D_veqm_r_times_pD (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_D_veqm_r_times_pD(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_D_veqm_pD (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_D_veqm_pD(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_D_xeq_r_times_D (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_D_xeq_r_times_D(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_D_xeq_D (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_D_xeq_D(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_D_xeq_r_times_pD (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_D_xeq_r_times_pD(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_D_xeq_pD (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_D_xeq_pD(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_D_xpeq_r_times_D (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_D_xpeq_r_times_D(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_D_xpeq_D (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_D_xpeq_D(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_D_xpeq_r_times_pD (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_D_xpeq_r_times_pD(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_D_xpeq_pD (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_D_xpeq_pD(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_D_xmeq_r_times_D (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_D_xmeq_r_times_D(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_D_xmeq_D (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_D_xmeq_D(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_D_xmeq_r_times_pD (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_D_xmeq_r_times_pD(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_D_xmeq_pD (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_D_xmeq_pD(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_D_xeqm_r_times_D (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_D_xeqm_r_times_D(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_D_xeqm_D (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_D_xeqm_D(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_D_xeqm_r_times_pD (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_D_xeqm_r_times_pD(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_D_xeqm_pD (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_D_xeqm_pD(int nc, void * r, void * a, int * index, int n);
/* ---- norm2: replaces the FN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_FN_r_veq_norm2_D (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_FN_r_veq_norm2_D(int nc, QLA_F_Real * r, void * a, int n);
/* replaces QLA_FN_r_veq_norm2_pD (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_FN_r_veq_norm2_pD(int nc, QLA_F_Real * r, void * a, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_veq_D_dot_D (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_veq_D_dot_D(int nc, QLA_F_Complex * r, void * a, void * b, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_veq_re_D_dot_D (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_veq_re_D_dot_D(int nc, QLA_F_Real * r, void * a, void * b, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_veq_D_dot_pD (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_veq_D_dot_pD(int nc, QLA_F_Complex * r, void * a, void * b, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_veq_re_D_dot_pD (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_veq_re_D_dot_pD(int nc, QLA_F_Real * r, void * a, void * b, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_veq_pD_dot_D (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_veq_pD_dot_D(int nc, QLA_F_Complex * r, void * a, void * b, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_veq_re_pD_dot_D (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_veq_re_pD_dot_D(int nc, QLA_F_Real * r, void * a, void * b, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_veq_pD_dot_pD (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_veq_pD_dot_pD(int nc, QLA_F_Complex * r, void * a, void * b, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_veq_re_pD_dot_pD (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_veq_re_pD_dot_pD(int nc, QLA_F_Real * r, void * a, void * b, int n);
/* ---- norm2: replaces the FN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_FN_r_xeq_norm2_D (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_FN_r_xeq_norm2_D(int nc, QLA_F_Real * r, void * a, int * index, int n);
/* replaces QLA_FN_r_xeq_norm2_pD (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_FN_r_xeq_norm2_pD(int nc, QLA_F_Real * r, void * a, int * index, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_xeq_D_dot_D (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_xeq_D_dot_D(int nc, QLA_F_Complex * r, void * a, void * b, int * index, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_xeq_re_D_dot_D (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_xeq_re_D_dot_D(int nc, QLA_F_Real * r, void * a, void * b, int * index, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_xeq_D_dot_pD (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_xeq_D_dot_pD(int nc, QLA_F_Complex * r, void * a, void * b, int * index, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_xeq_re_D_dot_pD (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_xeq_re_D_dot_pD(int nc, QLA_F_Real * r, void * a, void * b, int * index, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_xeq_pD_dot_D (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_xeq_pD_dot_D(int nc, QLA_F_Complex * r, void * a, void * b, int * index, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_xeq_re_pD_dot_D (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_xeq_re_pD_dot_D(int nc, QLA_F_Real * r, void * a, void * b, int * index, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_xeq_pD_dot_pD (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_xeq_pD_dot_pD(int nc, QLA_F_Complex * r, void * a, void * b, int * index, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_xeq_re_pD_dot_pD (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_xeq_re_pD_dot_pD(int nc, QLA_F_Real * r, void * a, void * b, int * index, int n);
/* ---- lmult: replaces the FN functions emitted by lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix) */
/* replaces QLA_FN_M_veq_M_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veq_M_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_M_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veq_M_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_M_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veq_M_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_M_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veq_M_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_Ma_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veq_Ma_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_Ma_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veq_Ma_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_Ma_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veq_Ma_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_Ma_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veq_Ma_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_pM_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veq_pM_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_pM_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veq_pM_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_pM_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veq_pM_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_pM_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veq_pM_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_pMa_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veq_pMa_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_pMa_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veq_pMa_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_pMa_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veq_pMa_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_pMa_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veq_pMa_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_M_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vpeq_M_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_M_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vpeq_M_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_M_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vpeq_M_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_M_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vpeq_M_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_Ma_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vpeq_Ma_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_Ma_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vpeq_Ma_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_Ma_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vpeq_Ma_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_Ma_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vpeq_Ma_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_pM_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vpeq_pM_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_pM_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vpeq_pM_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_pM_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vpeq_pM_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_pM_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vpeq_pM_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_pMa_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vpeq_pMa_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_pMa_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vpeq_pMa_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_pMa_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vpeq_pMa_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_pMa_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vpeq_pMa_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_M_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vmeq_M_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_M_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vmeq_M_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_M_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vmeq_M_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_M_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vmeq_M_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_Ma_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vmeq_Ma_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_Ma_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vmeq_Ma_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_Ma_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vmeq_Ma_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_Ma_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vmeq_Ma_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_pM_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vmeq_pM_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_pM_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vmeq_pM_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_pM_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vmeq_pM_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_pM_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vmeq_pM_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_pMa_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vmeq_pMa_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_pMa_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vmeq_pMa_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_pMa_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vmeq_pMa_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_pMa_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_vmeq_pMa_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veqm_M_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veqm_M_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veqm_M_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veqm_M_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veqm_M_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veqm_M_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veqm_M_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veqm_M_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veqm_Ma_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veqm_Ma_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veqm_Ma_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veqm_Ma_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veqm_Ma_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veqm_Ma_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veqm_Ma_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veqm_Ma_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veqm_pM_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veqm_pM_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veqm_pM_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veqm_pM_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veqm_pM_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veqm_pM_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veqm_pM_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veqm_pM_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veqm_pMa_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veqm_pMa_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veqm_pMa_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veqm_pMa_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veqm_pMa_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veqm_pMa_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veqm_pMa_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_veqm_pMa_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_xeq_M_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeq_M_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_M_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeq_M_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_M_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeq_M_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_M_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeq_M_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_Ma_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeq_Ma_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_Ma_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeq_Ma_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_Ma_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeq_Ma_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_Ma_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeq_Ma_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pM_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeq_pM_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pM_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeq_pM_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pM_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeq_pM_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pM_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeq_pM_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pMa_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeq_pMa_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pMa_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeq_pMa_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pMa_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeq_pMa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pMa_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeq_pMa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_M_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xpeq_M_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_M_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xpeq_M_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_M_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xpeq_M_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_M_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xpeq_M_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_Ma_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xpeq_Ma_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_Ma_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xpeq_Ma_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_Ma_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xpeq_Ma_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_Ma_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xpeq_Ma_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_pM_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xpeq_pM_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_pM_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xpeq_pM_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_pM_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xpeq_pM_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_pM_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xpeq_pM_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_pMa_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xpeq_pMa_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_pMa_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xpeq_pMa_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_pMa_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xpeq_pMa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_pMa_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xpeq_pMa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_M_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xmeq_M_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_M_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xmeq_M_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_M_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xmeq_M_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_M_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xmeq_M_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_Ma_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xmeq_Ma_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_Ma_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xmeq_Ma_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_Ma_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xmeq_Ma_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_Ma_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xmeq_Ma_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_pM_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xmeq_pM_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_pM_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xmeq_pM_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_pM_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xmeq_pM_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_pM_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xmeq_pM_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_pMa_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xmeq_pMa_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_pMa_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xmeq_pMa_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_pMa_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xmeq_pMa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_pMa_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xmeq_pMa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_M_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeqm_M_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_M_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeqm_M_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_M_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeqm_M_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_M_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeqm_M_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_Ma_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeqm_Ma_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_Ma_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeqm_Ma_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_Ma_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeqm_Ma_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_Ma_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeqm_Ma_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_pM_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeqm_pM_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_pM_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeqm_pM_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_pM_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeqm_pM_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_pM_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeqm_pM_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_pMa_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeqm_pMa_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_pMa_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeqm_pMa_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_pMa_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeqm_pMa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_pMa_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_FN_M_xeqm_pMa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_eq_M_times_xM (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_M_eq_M_times_xM(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_M_eq_Ma_times_xM (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_M_eq_Ma_times_xM(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_M_peq_M_times_xM (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_M_peq_M_times_xM(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_M_peq_Ma_times_xM (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_M_peq_Ma_times_xM(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_M_meq_M_times_xM (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_M_meq_M_times_xM(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_M_meq_Ma_times_xM (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_M_meq_Ma_times_xM(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_M_eqm_M_times_xM (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_M_eqm_M_times_xM(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_FN_M_eqm_Ma_times_xM (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_FN_M_eqm_Ma_times_xM(int nc, void * r, void * a, void * b, int * jb, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_M_veq_r_times_M (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_M_veq_r_times_M(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_M_veq_M (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_M_veq_M(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_M_veq_r_times_pM (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_M_veq_r_times_pM(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_M_veq_pM (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_M_veq_pM(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_M_vpeq_r_times_M (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_M_vpeq_r_times_M(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_M_vpeq_M (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_M_vpeq_M(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_M_vpeq_r_times_pM (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_M_vpeq_r_times_pM(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_M_vpeq_pM (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_M_vpeq_pM(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_M_vmeq_r_times_M (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_M_vmeq_r_times_M(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_M_vmeq_M (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_M_vmeq_M(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_M_vmeq_r_times_pM (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_M_vmeq_r_times_pM(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_M_vmeq_pM (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_M_vmeq_pM(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_M_veqm_r_times_M (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_M_veqm_r_times_M(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_M_veqm_M (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_M_veqm_M(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_M_veqm_r_times_pM (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_M_veqm_r_times_pM(int nc, void * r, QLA_F_Real * a, void * b, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_M_veqm_pM (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_M_veqm_pM(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_M_xeq_r_times_M (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_M_xeq_r_times_M(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_M_xeq_M (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_M_xeq_M(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_M_xeq_r_times_pM (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_M_xeq_r_times_pM(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_M_xeq_pM (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_M_xeq_pM(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_M_xpeq_r_times_M (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_M_xpeq_r_times_M(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_M_xpeq_M (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_M_xpeq_M(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_M_xpeq_r_times_pM (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_M_xpeq_r_times_pM(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_M_xpeq_pM (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_M_xpeq_pM(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_M_xmeq_r_times_M (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_M_xmeq_r_times_M(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_M_xmeq_M (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_M_xmeq_M(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_M_xmeq_r_times_pM (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_M_xmeq_r_times_pM(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_M_xmeq_pM (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_M_xmeq_pM(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_M_xeqm_r_times_M (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_M_xeqm_r_times_M(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_M_xeqm_M (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_M_xeqm_M(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_FN_M_xeqm_r_times_pM (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_FN_M_xeqm_r_times_pM(int nc, void * r, QLA_F_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the FN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_FN_M_xeqm_pM (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_FN_M_xeqm_pM(int nc, void * r, void * a, int * index, int n);
/* ---- norm2: replaces the FN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_FN_r_veq_norm2_M (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_FN_r_veq_norm2_M(int nc, QLA_F_Real * r, void * a, int n);
/* replaces QLA_FN_r_veq_norm2_pM (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_FN_r_veq_norm2_pM(int nc, QLA_F_Real * r, void * a, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_veq_M_dot_M (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_veq_M_dot_M(int nc, QLA_F_Complex * r, void * a, void * b, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_veq_re_M_dot_M (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_veq_re_M_dot_M(int nc, QLA_F_Real * r, void * a, void * b, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_veq_M_dot_pM (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_veq_M_dot_pM(int nc, QLA_F_Complex * r, void * a, void * b, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_veq_re_M_dot_pM (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_veq_re_M_dot_pM(int nc, QLA_F_Real * r, void * a, void * b, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_veq_pM_dot_M (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_veq_pM_dot_M(int nc, QLA_F_Complex * r, void * a, void * b, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_veq_re_pM_dot_M (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_veq_re_pM_dot_M(int nc, QLA_F_Real * r, void * a, void * b, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_veq_pM_dot_pM (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_veq_pM_dot_pM(int nc, QLA_F_Complex * r, void * a, void * b, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_veq_re_pM_dot_pM (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_veq_re_pM_dot_pM(int nc, QLA_F_Real * r, void * a, void * b, int n);
/* ---- norm2: replaces the FN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_FN_r_xeq_norm2_M (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_FN_r_xeq_norm2_M(int nc, QLA_F_Real * r, void * a, int * index, int n);
/* replaces QLA_FN_r_xeq_norm2_pM (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_FN_r_xeq_norm2_pM(int nc, QLA_F_Real * r, void * a, int * index, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_xeq_M_dot_M (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_xeq_M_dot_M(int nc, QLA_F_Complex * r, void * a, void * b, int * index, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_xeq_re_M_dot_M (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_xeq_re_M_dot_M(int nc, QLA_F_Real * r, void * a, void * b, int * index, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_xeq_M_dot_pM (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_xeq_M_dot_pM(int nc, QLA_F_Complex * r, void * a, void * b, int * index, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_xeq_re_M_dot_pM (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_xeq_re_M_dot_pM(int nc, QLA_F_Real * r, void * a, void * b, int * index, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_xeq_pM_dot_M (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_xeq_pM_dot_M(int nc, QLA_F_Complex * r, void * a, void * b, int * index, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_xeq_re_pM_dot_M (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_xeq_re_pM_dot_M(int nc, QLA_F_Real * r, void * a, void * b, int * index, int n);
/* ---- dot: replaces the FN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_FN_c_xeq_pM_dot_pM (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_FN_c_xeq_pM_dot_pM(int nc, QLA_F_Complex * r, void * a, void * b, int * index, int n);
/* ---- redot: replaces the FN functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_FN_r_xeq_re_pM_dot_pM (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_FN_r_xeq_re_pM_dot_pM(int nc, QLA_F_Real * r, void * a, void * b, int * index, int n);
/* ---- spproj: replaces the FN functions emitted by lib/perl/build_qla.pl:1087-1110 */
/* replaces QLA_FN_H_veq_spproj_D (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_FN_H_veq_spproj_D(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_FN_H_veq_spproj_pD (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_FN_H_veq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int n);
/* ---- sprecon: replaces the FN functions emitted by lib/perl/build_qla.pl:1112-1135 */
/* replaces QLA_FN_D_veq_sprecon_H (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_FN_D_veq_sprecon_H(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_FN_D_veq_sprecon_pH (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_FN_D_veq_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int n);
/* ---- spproj: replaces the FN functions emitted by lib/perl/build_qla.pl:1087-1110 */
/* replaces QLA_FN_H_vpeq_spproj_D (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_FN_H_vpeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_FN_H_vpeq_spproj_pD (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_FN_H_vpeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int n);
/* ---- sprecon: replaces the FN functions emitted by lib/perl/build_qla.pl:1112-1135 */
/* replaces QLA_FN_D_vpeq_sprecon_H (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_FN_D_vpeq_sprecon_H(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_FN_D_vpeq_sprecon_pH (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_FN_D_vpeq_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int n);
/* ---- spproj: replaces the FN functions emitted by lib/perl/build_qla.pl:1087-1110 */
/* replaces QLA_FN_H_vmeq_spproj_D (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_FN_H_vmeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_FN_H_vmeq_spproj_pD (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_FN_H_vmeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int n);
/* ---- sprecon: replaces the FN functions emitted by lib/perl/build_qla.pl:1112-1135 */
/* replaces QLA_FN_D_vmeq_sprecon_H (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_FN_D_vmeq_sprecon_H(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_FN_D_vmeq_sprecon_pH (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_FN_D_vmeq_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int n);
/* ---- spproj: replaces the FN functions emitted by lib/perl/build_qla.pl:1087-1110 */
/* replaces QLA_FN_H_veqm_spproj_D (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_FN_H_veqm_spproj_D(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_FN_H_veqm_spproj_pD (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_FN_H_veqm_spproj_pD(int nc, void * r, void * a, int mu, int sign, int n);
/* ---- sprecon: replaces the FN functions emitted by lib/perl/build_qla.pl:1112-1135 */
/* replaces QLA_FN_D_veqm_sprecon_H (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_FN_D_veqm_sprecon_H(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_FN_D_veqm_sprecon_pH (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_FN_D_veqm_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int n);
/* ---- mfunc: replaces the FN functions emitted by lib/perl/build_qla.pl:1000-1060 (matrix functions) */
/* replaces QLA_FN_M_veq_exp_M (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_FN_M_veq_exp_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_sqrt_M (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_FN_M_veq_sqrt_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_inverse_M (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_FN_M_veq_inverse_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_C_veq_det_M (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_FN_C_veq_det_M(int nc, QLA_F_Complex * r, void * a, int n);
/* ---- mfunc_ext: replaces the FN functions emitted by lib/perl/build_qla.pl:1022-1061 (matrix functions */
/* replaces QLA_FN_M_veq_invsqrt_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_veq_invsqrt_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_log_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_veq_log_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_expA_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_veq_expA_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_expTA_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_veq_expTA_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_sqrtPH_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_veq_sqrtPH_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_invsqrtPH_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_veq_invsqrtPH_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_veq_eigenvals_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_V_veq_eigenvals_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_veq_eigenvalsH_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_V_veq_eigenvalsH_M(int nc, void * r, void * a, int n);
/* ---- mfunc: replaces the FN functions emitted by lib/perl/build_qla.pl:1000-1060 (matrix functions) */
/* replaces QLA_FN_M_veq_exp_pM (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_FN_M_veq_exp_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_sqrt_pM (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_FN_M_veq_sqrt_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_inverse_pM (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_FN_M_veq_inverse_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_C_veq_det_pM (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_FN_C_veq_det_pM(int nc, QLA_F_Complex * r, void * a, int n);
/* ---- mfunc_ext: replaces the FN functions emitted by lib/perl/build_qla.pl:1022-1061 (matrix functions */
/* replaces QLA_FN_M_veq_invsqrt_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_veq_invsqrt_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_log_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_veq_log_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_expA_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_veq_expA_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_expTA_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_veq_expTA_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_sqrtPH_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_veq_sqrtPH_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_invsqrtPH_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_veq_invsqrtPH_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_veq_eigenvals_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_V_veq_eigenvals_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_veq_eigenvalsH_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_V_veq_eigenvalsH_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_veq_M_inverse_V (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_FN_V_veq_M_inverse_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veq_M_inverse_pV (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_FN_V_veq_M_inverse_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veq_pM_inverse_V (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_FN_V_veq_pM_inverse_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veq_pM_inverse_pV (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_FN_V_veq_pM_inverse_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_M_inverse_M (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_FN_M_veq_M_inverse_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_M_inverse_pM (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_FN_M_veq_M_inverse_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_pM_inverse_M (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_FN_M_veq_pM_inverse_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_pM_inverse_pM (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_FN_M_veq_pM_inverse_pM(int nc, void * r, void * a, void * b, int n);
/* ---- spproj: replaces the FN functions emitted by lib/perl/build_qla.pl:1087-1110 */
/* replaces QLA_FN_H_xeq_spproj_D (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_FN_H_xeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xeq_spproj_pD (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_FN_H_xeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* ---- sprecon: replaces the FN functions emitted by lib/perl/build_qla.pl:1112-1135 */
/* replaces QLA_FN_D_xeq_sprecon_H (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_FN_D_xeq_sprecon_H(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeq_sprecon_pH (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_FN_D_xeq_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* ---- spproj: replaces the FN functions emitted by lib/perl/build_qla.pl:1087-1110 */
/* replaces QLA_FN_H_xpeq_spproj_D (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_FN_H_xpeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xpeq_spproj_pD (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_FN_H_xpeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* ---- sprecon: replaces the FN functions emitted by lib/perl/build_qla.pl:1112-1135 */
/* replaces QLA_FN_D_xpeq_sprecon_H (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_FN_D_xpeq_sprecon_H(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xpeq_sprecon_pH (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_FN_D_xpeq_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* ---- spproj: replaces the FN functions emitted by lib/perl/build_qla.pl:1087-1110 */
/* replaces QLA_FN_H_xmeq_spproj_D (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_FN_H_xmeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xmeq_spproj_pD (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_FN_H_xmeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* ---- sprecon: replaces the FN functions emitted by lib/perl/build_qla.pl:1112-1135 */
/* replaces QLA_FN_D_xmeq_sprecon_H (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_FN_D_xmeq_sprecon_H(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xmeq_sprecon_pH (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_FN_D_xmeq_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* ---- spproj: replaces the FN functions emitted by lib/perl/build_qla.pl:1087-1110 */
/* replaces QLA_FN_H_xeqm_spproj_D (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_FN_H_xeqm_spproj_D(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xeqm_spproj_pD (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_FN_H_xeqm_spproj_pD(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* ---- sprecon: replaces the FN functions emitted by lib/perl/build_qla.pl:1112-1135 */
/* replaces QLA_FN_D_xeqm_sprecon_H (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_FN_D_xeqm_sprecon_H(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeqm_sprecon_pH (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_FN_D_xeqm_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* ---- mfunc: replaces the FN functions emitted by lib/perl/build_qla.pl:1000-1060 (matrix functions) */
/* replaces QLA_FN_M_xeq_exp_M (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_FN_M_xeq_exp_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_sqrt_M (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_FN_M_xeq_sqrt_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_inverse_M (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_FN_M_xeq_inverse_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_C_xeq_det_M (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_FN_C_xeq_det_M(int nc, QLA_F_Complex * r, void * a, int * index, int n);
/* ---- mfunc_ext: replaces the FN functions emitted by lib/perl/build_qla.pl:1022-1061 (matrix functions */
/* replaces QLA_FN_M_xeq_invsqrt_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_xeq_invsqrt_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_log_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_xeq_log_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_expA_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_xeq_expA_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_expTA_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_xeq_expTA_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_sqrtPH_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_xeq_sqrtPH_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_invsqrtPH_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_xeq_invsqrtPH_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xeq_eigenvals_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_V_xeq_eigenvals_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xeq_eigenvalsH_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_V_xeq_eigenvalsH_M(int nc, void * r, void * a, int * index, int n);
/* ---- mfunc: replaces the FN functions emitted by lib/perl/build_qla.pl:1000-1060 (matrix functions) */
/* replaces QLA_FN_M_xeq_exp_pM (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_FN_M_xeq_exp_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_sqrt_pM (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_FN_M_xeq_sqrt_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_inverse_pM (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_FN_M_xeq_inverse_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_C_xeq_det_pM (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_FN_C_xeq_det_pM(int nc, QLA_F_Complex * r, void * a, int * index, int n);
/* ---- mfunc_ext: replaces the FN functions emitted by lib/perl/build_qla.pl:1022-1061 (matrix functions */
/* replaces QLA_FN_M_xeq_invsqrt_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_xeq_invsqrt_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_log_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_xeq_log_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_expA_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_xeq_expA_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_expTA_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_xeq_expTA_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_sqrtPH_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_xeq_sqrtPH_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_invsqrtPH_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_M_xeq_invsqrtPH_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xeq_eigenvals_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_V_xeq_eigenvals_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xeq_eigenvalsH_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_FN_V_xeq_eigenvalsH_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xeq_M_inverse_V (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_FN_V_xeq_M_inverse_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_M_inverse_pV (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_FN_V_xeq_M_inverse_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_pM_inverse_V (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_FN_V_xeq_pM_inverse_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_pM_inverse_pV (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_FN_V_xeq_pM_inverse_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_M_inverse_M (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_FN_M_xeq_M_inverse_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_M_inverse_pM (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_FN_M_xeq_M_inverse_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pM_inverse_M (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_FN_M_xeq_pM_inverse_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pM_inverse_pM (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_FN_M_xeq_pM_inverse_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* ---- hop: replaces the FN functions emitted by lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix) */
/* replaces QLA_FN_H_veq_spproj_M_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_veq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_veq_spproj_M_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_veq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veq_spproj_M_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veq_spproj_M_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veq_sprecon_M_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veq_sprecon_M_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veq_sprecon_M_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veq_sprecon_M_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_veq_spproj_Ma_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_veq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_veq_spproj_Ma_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_veq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veq_spproj_Ma_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veq_spproj_Ma_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veq_sprecon_Ma_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veq_sprecon_Ma_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veq_sprecon_Ma_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veq_sprecon_Ma_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_veq_spproj_pM_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_veq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_veq_spproj_pM_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_veq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veq_spproj_pM_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veq_spproj_pM_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veq_sprecon_pM_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veq_sprecon_pM_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veq_sprecon_pM_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veq_sprecon_pM_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_veq_spproj_pMa_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_veq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_veq_spproj_pMa_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_veq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veq_spproj_pMa_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veq_spproj_pMa_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veq_sprecon_pMa_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veq_sprecon_pMa_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veq_sprecon_pMa_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veq_sprecon_pMa_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veq_spproj_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veq_spproj_D(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_FN_D_veq_spproj_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_FN_H_vpeq_spproj_M_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_vpeq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_vpeq_spproj_M_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_vpeq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vpeq_spproj_M_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vpeq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vpeq_spproj_M_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vpeq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vpeq_sprecon_M_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vpeq_sprecon_M_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vpeq_sprecon_M_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vpeq_sprecon_M_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_vpeq_spproj_Ma_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_vpeq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_vpeq_spproj_Ma_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_vpeq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vpeq_spproj_Ma_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vpeq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vpeq_spproj_Ma_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vpeq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vpeq_sprecon_Ma_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vpeq_sprecon_Ma_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vpeq_sprecon_Ma_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vpeq_sprecon_Ma_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_vpeq_spproj_pM_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_vpeq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_vpeq_spproj_pM_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_vpeq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vpeq_spproj_pM_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vpeq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vpeq_spproj_pM_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vpeq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vpeq_sprecon_pM_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vpeq_sprecon_pM_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vpeq_sprecon_pM_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vpeq_sprecon_pM_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_vpeq_spproj_pMa_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_vpeq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_vpeq_spproj_pMa_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_vpeq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vpeq_spproj_pMa_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vpeq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vpeq_spproj_pMa_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vpeq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vpeq_sprecon_pMa_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vpeq_sprecon_pMa_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vpeq_sprecon_pMa_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vpeq_sprecon_pMa_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vpeq_spproj_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vpeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_FN_D_vpeq_spproj_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vpeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_FN_H_vmeq_spproj_M_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_vmeq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_vmeq_spproj_M_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_vmeq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vmeq_spproj_M_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vmeq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vmeq_spproj_M_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vmeq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vmeq_sprecon_M_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vmeq_sprecon_M_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vmeq_sprecon_M_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vmeq_sprecon_M_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_vmeq_spproj_Ma_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_vmeq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_vmeq_spproj_Ma_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_vmeq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vmeq_spproj_Ma_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vmeq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vmeq_spproj_Ma_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vmeq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vmeq_sprecon_Ma_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vmeq_sprecon_Ma_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vmeq_sprecon_Ma_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vmeq_sprecon_Ma_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_vmeq_spproj_pM_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_vmeq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_vmeq_spproj_pM_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_vmeq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vmeq_spproj_pM_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vmeq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vmeq_spproj_pM_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vmeq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vmeq_sprecon_pM_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vmeq_sprecon_pM_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vmeq_sprecon_pM_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vmeq_sprecon_pM_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_vmeq_spproj_pMa_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_vmeq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_vmeq_spproj_pMa_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_vmeq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vmeq_spproj_pMa_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vmeq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vmeq_spproj_pMa_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vmeq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vmeq_sprecon_pMa_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vmeq_sprecon_pMa_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vmeq_sprecon_pMa_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vmeq_sprecon_pMa_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_vmeq_spproj_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vmeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_FN_D_vmeq_spproj_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_vmeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_FN_H_veqm_spproj_M_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_veqm_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_veqm_spproj_M_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_veqm_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veqm_spproj_M_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veqm_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veqm_spproj_M_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veqm_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veqm_sprecon_M_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veqm_sprecon_M_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veqm_sprecon_M_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veqm_sprecon_M_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_veqm_spproj_Ma_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_veqm_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_veqm_spproj_Ma_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_veqm_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veqm_spproj_Ma_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veqm_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veqm_spproj_Ma_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veqm_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veqm_sprecon_Ma_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veqm_sprecon_Ma_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veqm_sprecon_Ma_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veqm_sprecon_Ma_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_veqm_spproj_pM_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_veqm_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_veqm_spproj_pM_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_veqm_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veqm_spproj_pM_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veqm_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veqm_spproj_pM_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veqm_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veqm_sprecon_pM_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veqm_sprecon_pM_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veqm_sprecon_pM_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veqm_sprecon_pM_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_veqm_spproj_pMa_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_veqm_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_H_veqm_spproj_pMa_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_veqm_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veqm_spproj_pMa_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veqm_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veqm_spproj_pMa_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veqm_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veqm_sprecon_pMa_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veqm_sprecon_pMa_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veqm_sprecon_pMa_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veqm_sprecon_pMa_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int n);
/* replaces QLA_FN_D_veqm_spproj_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veqm_spproj_D(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_FN_D_veqm_spproj_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_veqm_spproj_pD(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_FN_H_xeq_spproj_M_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xeq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xeq_spproj_M_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xeq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeq_spproj_M_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeq_spproj_M_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeq_sprecon_M_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeq_sprecon_M_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeq_sprecon_M_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeq_sprecon_M_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xeq_spproj_Ma_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xeq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xeq_spproj_Ma_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xeq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeq_spproj_Ma_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeq_spproj_Ma_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeq_sprecon_Ma_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeq_sprecon_Ma_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeq_sprecon_Ma_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeq_sprecon_Ma_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xeq_spproj_pM_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xeq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xeq_spproj_pM_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xeq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeq_spproj_pM_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeq_spproj_pM_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeq_sprecon_pM_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeq_sprecon_pM_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeq_sprecon_pM_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeq_sprecon_pM_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xeq_spproj_pMa_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xeq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xeq_spproj_pMa_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xeq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeq_spproj_pMa_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeq_spproj_pMa_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeq_sprecon_pMa_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeq_sprecon_pMa_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeq_sprecon_pMa_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeq_sprecon_pMa_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeq_spproj_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeq_spproj_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xpeq_spproj_M_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xpeq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xpeq_spproj_M_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xpeq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xpeq_spproj_M_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xpeq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xpeq_spproj_M_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xpeq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xpeq_sprecon_M_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xpeq_sprecon_M_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xpeq_sprecon_M_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xpeq_sprecon_M_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xpeq_spproj_Ma_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xpeq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xpeq_spproj_Ma_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xpeq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xpeq_spproj_Ma_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xpeq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xpeq_spproj_Ma_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xpeq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xpeq_sprecon_Ma_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xpeq_sprecon_Ma_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xpeq_sprecon_Ma_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xpeq_sprecon_Ma_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xpeq_spproj_pM_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xpeq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xpeq_spproj_pM_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xpeq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xpeq_spproj_pM_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xpeq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xpeq_spproj_pM_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xpeq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xpeq_sprecon_pM_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xpeq_sprecon_pM_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xpeq_sprecon_pM_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xpeq_sprecon_pM_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xpeq_spproj_pMa_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xpeq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xpeq_spproj_pMa_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xpeq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xpeq_spproj_pMa_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xpeq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xpeq_spproj_pMa_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xpeq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xpeq_sprecon_pMa_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xpeq_sprecon_pMa_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xpeq_sprecon_pMa_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xpeq_sprecon_pMa_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xpeq_spproj_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xpeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xpeq_spproj_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xpeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xmeq_spproj_M_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xmeq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xmeq_spproj_M_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xmeq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xmeq_spproj_M_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xmeq_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xmeq_spproj_M_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xmeq_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xmeq_sprecon_M_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xmeq_sprecon_M_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xmeq_sprecon_M_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xmeq_sprecon_M_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xmeq_spproj_Ma_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xmeq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xmeq_spproj_Ma_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xmeq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xmeq_spproj_Ma_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xmeq_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xmeq_spproj_Ma_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xmeq_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xmeq_sprecon_Ma_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xmeq_sprecon_Ma_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xmeq_sprecon_Ma_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xmeq_sprecon_Ma_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xmeq_spproj_pM_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xmeq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xmeq_spproj_pM_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xmeq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xmeq_spproj_pM_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xmeq_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xmeq_spproj_pM_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xmeq_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xmeq_sprecon_pM_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xmeq_sprecon_pM_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xmeq_sprecon_pM_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xmeq_sprecon_pM_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xmeq_spproj_pMa_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xmeq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xmeq_spproj_pMa_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xmeq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xmeq_spproj_pMa_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xmeq_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xmeq_spproj_pMa_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xmeq_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xmeq_sprecon_pMa_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xmeq_sprecon_pMa_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xmeq_sprecon_pMa_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xmeq_sprecon_pMa_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xmeq_spproj_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xmeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xmeq_spproj_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xmeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xeqm_spproj_M_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xeqm_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xeqm_spproj_M_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xeqm_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeqm_spproj_M_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeqm_spproj_M_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeqm_spproj_M_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeqm_spproj_M_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeqm_sprecon_M_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeqm_sprecon_M_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeqm_sprecon_M_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeqm_sprecon_M_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xeqm_spproj_Ma_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xeqm_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xeqm_spproj_Ma_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xeqm_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeqm_spproj_Ma_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeqm_spproj_Ma_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeqm_spproj_Ma_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeqm_spproj_Ma_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeqm_sprecon_Ma_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeqm_sprecon_Ma_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeqm_sprecon_Ma_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeqm_sprecon_Ma_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xeqm_spproj_pM_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xeqm_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xeqm_spproj_pM_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xeqm_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeqm_spproj_pM_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeqm_spproj_pM_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeqm_spproj_pM_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeqm_spproj_pM_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeqm_sprecon_pM_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeqm_sprecon_pM_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeqm_sprecon_pM_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeqm_sprecon_pM_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xeqm_spproj_pMa_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xeqm_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_xeqm_spproj_pMa_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_H_xeqm_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeqm_spproj_pMa_times_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeqm_spproj_pMa_times_D(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeqm_spproj_pMa_times_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeqm_spproj_pMa_times_pD(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeqm_sprecon_pMa_times_H (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeqm_sprecon_pMa_times_H(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeqm_sprecon_pMa_times_pH (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeqm_sprecon_pMa_times_pH(int nc, void * r, void * a, void * b, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeqm_spproj_D (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeqm_spproj_D(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_FN_D_xeqm_spproj_pD (lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336) */
void QLA_FN_D_xeqm_spproj_pD(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_FN_H_eq_spproj_M_times_xD (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_H_eq_spproj_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* replaces QLA_FN_D_eq_spproj_M_times_xD (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_D_eq_spproj_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* replaces QLA_FN_D_eq_sprecon_M_times_xH (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_D_eq_sprecon_M_times_xH(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* replaces QLA_FN_H_eq_spproj_Ma_times_xD (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_H_eq_spproj_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* replaces QLA_FN_D_eq_spproj_Ma_times_xD (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_D_eq_spproj_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* replaces QLA_FN_D_eq_sprecon_Ma_times_xH (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_D_eq_sprecon_Ma_times_xH(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* replaces QLA_FN_H_peq_spproj_M_times_xD (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_H_peq_spproj_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* replaces QLA_FN_D_peq_spproj_M_times_xD (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_D_peq_spproj_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* replaces QLA_FN_D_peq_sprecon_M_times_xH (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_D_peq_sprecon_M_times_xH(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* replaces QLA_FN_H_peq_spproj_Ma_times_xD (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_H_peq_spproj_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* replaces QLA_FN_D_peq_spproj_Ma_times_xD (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_D_peq_spproj_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* replaces QLA_FN_D_peq_sprecon_Ma_times_xH (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_D_peq_sprecon_Ma_times_xH(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* replaces QLA_FN_H_meq_spproj_M_times_xD (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_H_meq_spproj_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* replaces QLA_FN_D_meq_spproj_M_times_xD (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_D_meq_spproj_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* replaces QLA_FN_D_meq_sprecon_M_times_xH (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_D_meq_sprecon_M_times_xH(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* replaces QLA_FN_H_meq_spproj_Ma_times_xD (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_H_meq_spproj_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* replaces QLA_FN_D_meq_spproj_Ma_times_xD (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_D_meq_spproj_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* replaces QLA_FN_D_meq_sprecon_Ma_times_xH (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_D_meq_sprecon_Ma_times_xH(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* replaces QLA_FN_H_eqm_spproj_M_times_xD (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_H_eqm_spproj_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* replaces QLA_FN_D_eqm_spproj_M_times_xD (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_D_eqm_spproj_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* replaces QLA_FN_D_eqm_sprecon_M_times_xH (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_D_eqm_sprecon_M_times_xH(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* replaces QLA_FN_H_eqm_spproj_Ma_times_xD (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_H_eqm_spproj_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* replaces QLA_FN_D_eqm_spproj_Ma_times_xD (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_D_eqm_spproj_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* replaces QLA_FN_D_eqm_sprecon_Ma_times_xH (doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)) */
void QLA_FN_D_eqm_sprecon_Ma_times_xH(int nc, void * r, void * a, void * b, int * jb, int mu, int sign, int n);
/* ---- ewise_v: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1335 (constant multiples of a field) */
/* replaces QLA_FN_V_veq_c_times_V (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_V_veq_c_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_veq_c_times_pV (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_V_veq_c_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_veq_C_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veq_C_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_veq_C_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veq_C_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_veq_pC_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veq_pC_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_veq_pC_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veq_pC_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_veq_Ca_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veq_Ca_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_veq_Ca_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veq_Ca_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_veq_pCa_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veq_pCa_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_veq_pCa_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veq_pCa_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_veq_R_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veq_R_times_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_veq_R_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veq_R_times_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_veq_pR_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veq_pR_times_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_veq_pR_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veq_pR_times_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_veq_conj_V (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_veq_conj_V(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_veq_conj_pV (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_veq_conj_pV(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_veq_i_V (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_veq_i_V(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_veq_i_pV (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_veq_i_pV(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_vpeq_c_times_V (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_V_vpeq_c_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_vpeq_c_times_pV (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_V_vpeq_c_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_vpeq_C_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vpeq_C_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_vpeq_C_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vpeq_C_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_vpeq_pC_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vpeq_pC_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_vpeq_pC_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vpeq_pC_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_vpeq_Ca_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vpeq_Ca_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_vpeq_Ca_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vpeq_Ca_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_vpeq_pCa_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vpeq_pCa_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_vpeq_pCa_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vpeq_pCa_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_vpeq_R_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vpeq_R_times_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_vpeq_R_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vpeq_R_times_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_vpeq_pR_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vpeq_pR_times_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_vpeq_pR_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vpeq_pR_times_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_vpeq_conj_V (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_vpeq_conj_V(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_vpeq_conj_pV (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_vpeq_conj_pV(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_vpeq_i_V (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_vpeq_i_V(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_vpeq_i_pV (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_vpeq_i_pV(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_vmeq_c_times_V (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_V_vmeq_c_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_vmeq_c_times_pV (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_V_vmeq_c_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_vmeq_C_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vmeq_C_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_vmeq_C_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vmeq_C_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_vmeq_pC_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vmeq_pC_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_vmeq_pC_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vmeq_pC_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_vmeq_Ca_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vmeq_Ca_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_vmeq_Ca_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vmeq_Ca_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_vmeq_pCa_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vmeq_pCa_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_vmeq_pCa_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vmeq_pCa_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_vmeq_R_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vmeq_R_times_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_vmeq_R_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vmeq_R_times_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_vmeq_pR_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vmeq_pR_times_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_vmeq_pR_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_vmeq_pR_times_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_vmeq_conj_V (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_vmeq_conj_V(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_vmeq_conj_pV (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_vmeq_conj_pV(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_vmeq_i_V (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_vmeq_i_V(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_vmeq_i_pV (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_vmeq_i_pV(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_veqm_c_times_V (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_V_veqm_c_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_veqm_c_times_pV (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_V_veqm_c_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_veqm_C_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veqm_C_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_veqm_C_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veqm_C_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_veqm_pC_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veqm_pC_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_veqm_pC_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veqm_pC_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_veqm_Ca_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veqm_Ca_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_veqm_Ca_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veqm_Ca_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_veqm_pCa_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veqm_pCa_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_veqm_pCa_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veqm_pCa_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_veqm_R_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veqm_R_times_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_veqm_R_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veqm_R_times_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_V_veqm_pR_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veqm_pR_times_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_veqm_pR_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_veqm_pR_times_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_V_veqm_conj_V (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_veqm_conj_V(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_veqm_conj_pV (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_veqm_conj_pV(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_veqm_i_V (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_veqm_i_V(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_veqm_i_pV (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_veqm_i_pV(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_veq_V_plus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_V_plus_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veq_r_times_V_plus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_r_times_V_plus_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_V_veq_c_times_V_plus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_c_times_V_plus_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_V_veq_V_minus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_V_minus_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veq_r_times_V_minus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_r_times_V_minus_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_V_veq_c_times_V_minus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_c_times_V_minus_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_V_veq_V_plus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_V_plus_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veq_r_times_V_plus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_r_times_V_plus_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_V_veq_c_times_V_plus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_c_times_V_plus_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_V_veq_V_minus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_V_minus_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veq_r_times_V_minus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_r_times_V_minus_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_V_veq_c_times_V_minus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_c_times_V_minus_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_V_veq_pV_plus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_pV_plus_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veq_r_times_pV_plus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_r_times_pV_plus_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_V_veq_c_times_pV_plus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_c_times_pV_plus_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_V_veq_pV_minus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_pV_minus_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veq_r_times_pV_minus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_r_times_pV_minus_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_V_veq_c_times_pV_minus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_c_times_pV_minus_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_V_veq_pV_plus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_pV_plus_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veq_r_times_pV_plus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_r_times_pV_plus_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_V_veq_c_times_pV_plus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_c_times_pV_plus_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_V_veq_pV_minus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_pV_minus_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_V_veq_r_times_pV_minus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_r_times_pV_minus_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_V_veq_c_times_pV_minus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_veq_c_times_pV_minus_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_V_xeq_c_times_V (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_V_xeq_c_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_c_times_pV (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_V_xeq_c_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_C_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeq_C_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_C_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeq_C_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_pC_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeq_pC_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_pC_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeq_pC_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_Ca_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeq_Ca_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_Ca_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeq_Ca_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_pCa_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeq_pCa_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_pCa_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeq_pCa_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_R_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeq_R_times_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_R_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeq_R_times_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_pR_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeq_pR_times_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_pR_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeq_pR_times_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_conj_V (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_xeq_conj_V(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xeq_conj_pV (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_xeq_conj_pV(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xeq_i_V (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_xeq_i_V(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xeq_i_pV (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_xeq_i_pV(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xpeq_c_times_V (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_V_xpeq_c_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xpeq_c_times_pV (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_V_xpeq_c_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xpeq_C_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xpeq_C_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xpeq_C_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xpeq_C_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xpeq_pC_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xpeq_pC_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xpeq_pC_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xpeq_pC_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xpeq_Ca_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xpeq_Ca_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xpeq_Ca_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xpeq_Ca_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xpeq_pCa_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xpeq_pCa_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xpeq_pCa_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xpeq_pCa_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xpeq_R_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xpeq_R_times_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xpeq_R_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xpeq_R_times_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xpeq_pR_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xpeq_pR_times_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xpeq_pR_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xpeq_pR_times_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xpeq_conj_V (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_xpeq_conj_V(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xpeq_conj_pV (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_xpeq_conj_pV(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xpeq_i_V (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_xpeq_i_V(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xpeq_i_pV (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_xpeq_i_pV(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xmeq_c_times_V (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_V_xmeq_c_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xmeq_c_times_pV (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_V_xmeq_c_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xmeq_C_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xmeq_C_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xmeq_C_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xmeq_C_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xmeq_pC_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xmeq_pC_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xmeq_pC_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xmeq_pC_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xmeq_Ca_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xmeq_Ca_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xmeq_Ca_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xmeq_Ca_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xmeq_pCa_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xmeq_pCa_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xmeq_pCa_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xmeq_pCa_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xmeq_R_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xmeq_R_times_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xmeq_R_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xmeq_R_times_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xmeq_pR_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xmeq_pR_times_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xmeq_pR_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xmeq_pR_times_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xmeq_conj_V (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_xmeq_conj_V(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xmeq_conj_pV (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_xmeq_conj_pV(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xmeq_i_V (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_xmeq_i_V(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xmeq_i_pV (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_xmeq_i_pV(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xeqm_c_times_V (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_V_xeqm_c_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeqm_c_times_pV (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_V_xeqm_c_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeqm_C_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeqm_C_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeqm_C_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeqm_C_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeqm_pC_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeqm_pC_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeqm_pC_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeqm_pC_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeqm_Ca_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeqm_Ca_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeqm_Ca_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeqm_Ca_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeqm_pCa_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeqm_pCa_times_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeqm_pCa_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeqm_pCa_times_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeqm_R_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeqm_R_times_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeqm_R_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeqm_R_times_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeqm_pR_times_V (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeqm_pR_times_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeqm_pR_times_pV (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_V_xeqm_pR_times_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeqm_conj_V (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_xeqm_conj_V(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xeqm_conj_pV (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_xeqm_conj_pV(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xeqm_i_V (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_xeqm_i_V(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xeqm_i_pV (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_V_xeqm_i_pV(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xeq_V_plus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_V_plus_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_r_times_V_plus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_r_times_V_plus_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_V_xeq_c_times_V_plus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_c_times_V_plus_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_V_xeq_V_minus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_V_minus_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_r_times_V_minus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_r_times_V_minus_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_V_xeq_c_times_V_minus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_c_times_V_minus_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_V_xeq_V_plus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_V_plus_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_r_times_V_plus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_r_times_V_plus_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_V_xeq_c_times_V_plus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_c_times_V_plus_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_V_xeq_V_minus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_V_minus_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_r_times_V_minus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_r_times_V_minus_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_V_xeq_c_times_V_minus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_c_times_V_minus_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_V_xeq_pV_plus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_pV_plus_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_r_times_pV_plus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_r_times_pV_plus_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_V_xeq_c_times_pV_plus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_c_times_pV_plus_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_V_xeq_pV_minus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_pV_minus_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_r_times_pV_minus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_r_times_pV_minus_V(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_V_xeq_c_times_pV_minus_V (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_c_times_pV_minus_V(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_V_xeq_pV_plus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_pV_plus_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_r_times_pV_plus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_r_times_pV_plus_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_V_xeq_c_times_pV_plus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_c_times_pV_plus_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_V_xeq_pV_minus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_pV_minus_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_V_xeq_r_times_pV_minus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_r_times_pV_minus_pV(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_V_xeq_c_times_pV_minus_pV (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_V_xeq_c_times_pV_minus_pV(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* ---- ewise_h: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1335 (constant multiples of a field) */
/* replaces QLA_FN_H_veq_c_times_H (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_H_veq_c_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_veq_c_times_pH (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_H_veq_c_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_veq_C_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veq_C_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_veq_C_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veq_C_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_veq_pC_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veq_pC_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_veq_pC_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veq_pC_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_veq_Ca_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veq_Ca_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_veq_Ca_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veq_Ca_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_veq_pCa_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veq_pCa_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_veq_pCa_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veq_pCa_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_veq_R_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veq_R_times_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_veq_R_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veq_R_times_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_veq_pR_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veq_pR_times_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_veq_pR_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veq_pR_times_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_veq_conj_H (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_veq_conj_H(int nc, void * r, void * a, int n);
/* replaces QLA_FN_H_veq_conj_pH (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_veq_conj_pH(int nc, void * r, void * a, int n);
/* replaces QLA_FN_H_veq_i_H (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_veq_i_H(int nc, void * r, void * a, int n);
/* replaces QLA_FN_H_veq_i_pH (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_veq_i_pH(int nc, void * r, void * a, int n);
/* replaces QLA_FN_H_vpeq_c_times_H (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_H_vpeq_c_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_vpeq_c_times_pH (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_H_vpeq_c_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_vpeq_C_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vpeq_C_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_vpeq_C_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vpeq_C_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_vpeq_pC_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vpeq_pC_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_vpeq_pC_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vpeq_pC_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_vpeq_Ca_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vpeq_Ca_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_vpeq_Ca_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vpeq_Ca_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_vpeq_pCa_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vpeq_pCa_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_vpeq_pCa_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vpeq_pCa_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_vpeq_R_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vpeq_R_times_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_vpeq_R_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vpeq_R_times_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_vpeq_pR_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vpeq_pR_times_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_vpeq_pR_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vpeq_pR_times_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_vpeq_conj_H (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_vpeq_conj_H(int nc, void * r, void * a, int n);
/* replaces QLA_FN_H_vpeq_conj_pH (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_vpeq_conj_pH(int nc, void * r, void * a, int n);
/* replaces QLA_FN_H_vpeq_i_H (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_vpeq_i_H(int nc, void * r, void * a, int n);
/* replaces QLA_FN_H_vpeq_i_pH (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_vpeq_i_pH(int nc, void * r, void * a, int n);
/* replaces QLA_FN_H_vmeq_c_times_H (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_H_vmeq_c_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_vmeq_c_times_pH (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_H_vmeq_c_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_vmeq_C_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vmeq_C_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_vmeq_C_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vmeq_C_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_vmeq_pC_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vmeq_pC_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_vmeq_pC_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vmeq_pC_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_vmeq_Ca_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vmeq_Ca_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_vmeq_Ca_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vmeq_Ca_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_vmeq_pCa_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vmeq_pCa_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_vmeq_pCa_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vmeq_pCa_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_vmeq_R_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vmeq_R_times_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_vmeq_R_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vmeq_R_times_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_vmeq_pR_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vmeq_pR_times_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_vmeq_pR_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_vmeq_pR_times_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_vmeq_conj_H (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_vmeq_conj_H(int nc, void * r, void * a, int n);
/* replaces QLA_FN_H_vmeq_conj_pH (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_vmeq_conj_pH(int nc, void * r, void * a, int n);
/* replaces QLA_FN_H_vmeq_i_H (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_vmeq_i_H(int nc, void * r, void * a, int n);
/* replaces QLA_FN_H_vmeq_i_pH (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_vmeq_i_pH(int nc, void * r, void * a, int n);
/* replaces QLA_FN_H_veqm_c_times_H (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_H_veqm_c_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_veqm_c_times_pH (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_H_veqm_c_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_veqm_C_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veqm_C_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_veqm_C_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veqm_C_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_veqm_pC_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veqm_pC_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_veqm_pC_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veqm_pC_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_veqm_Ca_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veqm_Ca_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_veqm_Ca_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veqm_Ca_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_veqm_pCa_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veqm_pCa_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_veqm_pCa_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veqm_pCa_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_veqm_R_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veqm_R_times_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_veqm_R_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veqm_R_times_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_H_veqm_pR_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veqm_pR_times_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_veqm_pR_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_veqm_pR_times_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_H_veqm_conj_H (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_veqm_conj_H(int nc, void * r, void * a, int n);
/* replaces QLA_FN_H_veqm_conj_pH (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_veqm_conj_pH(int nc, void * r, void * a, int n);
/* replaces QLA_FN_H_veqm_i_H (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_veqm_i_H(int nc, void * r, void * a, int n);
/* replaces QLA_FN_H_veqm_i_pH (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_veqm_i_pH(int nc, void * r, void * a, int n);
/* replaces QLA_FN_H_veq_H_plus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_H_plus_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_veq_r_times_H_plus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_r_times_H_plus_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_H_veq_c_times_H_plus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_c_times_H_plus_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_H_veq_H_minus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_H_minus_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_veq_r_times_H_minus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_r_times_H_minus_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_H_veq_c_times_H_minus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_c_times_H_minus_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_H_veq_H_plus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_H_plus_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_veq_r_times_H_plus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_r_times_H_plus_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_H_veq_c_times_H_plus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_c_times_H_plus_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_H_veq_H_minus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_H_minus_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_veq_r_times_H_minus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_r_times_H_minus_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_H_veq_c_times_H_minus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_c_times_H_minus_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_H_veq_pH_plus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_pH_plus_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_veq_r_times_pH_plus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_r_times_pH_plus_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_H_veq_c_times_pH_plus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_c_times_pH_plus_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_H_veq_pH_minus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_pH_minus_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_veq_r_times_pH_minus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_r_times_pH_minus_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_H_veq_c_times_pH_minus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_c_times_pH_minus_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_H_veq_pH_plus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_pH_plus_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_veq_r_times_pH_plus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_r_times_pH_plus_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_H_veq_c_times_pH_plus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_c_times_pH_plus_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_H_veq_pH_minus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_pH_minus_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_H_veq_r_times_pH_minus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_r_times_pH_minus_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_H_veq_c_times_pH_minus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_veq_c_times_pH_minus_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_H_xeq_c_times_H (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_H_xeq_c_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_c_times_pH (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_H_xeq_c_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_C_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeq_C_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_C_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeq_C_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_pC_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeq_pC_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_pC_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeq_pC_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_Ca_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeq_Ca_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_Ca_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeq_Ca_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_pCa_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeq_pCa_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_pCa_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeq_pCa_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_R_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeq_R_times_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_R_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeq_R_times_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_pR_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeq_pR_times_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_pR_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeq_pR_times_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_conj_H (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_xeq_conj_H(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_H_xeq_conj_pH (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_xeq_conj_pH(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_H_xeq_i_H (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_xeq_i_H(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_H_xeq_i_pH (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_xeq_i_pH(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_H_xpeq_c_times_H (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_H_xpeq_c_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xpeq_c_times_pH (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_H_xpeq_c_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xpeq_C_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xpeq_C_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xpeq_C_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xpeq_C_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xpeq_pC_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xpeq_pC_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xpeq_pC_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xpeq_pC_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xpeq_Ca_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xpeq_Ca_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xpeq_Ca_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xpeq_Ca_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xpeq_pCa_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xpeq_pCa_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xpeq_pCa_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xpeq_pCa_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xpeq_R_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xpeq_R_times_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xpeq_R_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xpeq_R_times_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xpeq_pR_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xpeq_pR_times_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xpeq_pR_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xpeq_pR_times_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xpeq_conj_H (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_xpeq_conj_H(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_H_xpeq_conj_pH (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_xpeq_conj_pH(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_H_xpeq_i_H (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_xpeq_i_H(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_H_xpeq_i_pH (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_xpeq_i_pH(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_H_xmeq_c_times_H (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_H_xmeq_c_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xmeq_c_times_pH (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_H_xmeq_c_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xmeq_C_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xmeq_C_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xmeq_C_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xmeq_C_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xmeq_pC_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xmeq_pC_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xmeq_pC_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xmeq_pC_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xmeq_Ca_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xmeq_Ca_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xmeq_Ca_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xmeq_Ca_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xmeq_pCa_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xmeq_pCa_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xmeq_pCa_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xmeq_pCa_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xmeq_R_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xmeq_R_times_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xmeq_R_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xmeq_R_times_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xmeq_pR_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xmeq_pR_times_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xmeq_pR_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xmeq_pR_times_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xmeq_conj_H (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_xmeq_conj_H(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_H_xmeq_conj_pH (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_xmeq_conj_pH(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_H_xmeq_i_H (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_xmeq_i_H(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_H_xmeq_i_pH (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_xmeq_i_pH(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_H_xeqm_c_times_H (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_H_xeqm_c_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeqm_c_times_pH (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_H_xeqm_c_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeqm_C_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeqm_C_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeqm_C_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeqm_C_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeqm_pC_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeqm_pC_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeqm_pC_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeqm_pC_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeqm_Ca_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeqm_Ca_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeqm_Ca_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeqm_Ca_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeqm_pCa_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeqm_pCa_times_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeqm_pCa_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeqm_pCa_times_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeqm_R_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeqm_R_times_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeqm_R_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeqm_R_times_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeqm_pR_times_H (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeqm_pR_times_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeqm_pR_times_pH (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_H_xeqm_pR_times_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeqm_conj_H (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_xeqm_conj_H(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_H_xeqm_conj_pH (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_xeqm_conj_pH(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_H_xeqm_i_H (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_xeqm_i_H(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_H_xeqm_i_pH (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_H_xeqm_i_pH(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_H_xeq_H_plus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_H_plus_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_r_times_H_plus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_r_times_H_plus_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_H_xeq_c_times_H_plus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_c_times_H_plus_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_H_xeq_H_minus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_H_minus_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_r_times_H_minus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_r_times_H_minus_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_H_xeq_c_times_H_minus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_c_times_H_minus_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_H_xeq_H_plus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_H_plus_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_r_times_H_plus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_r_times_H_plus_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_H_xeq_c_times_H_plus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_c_times_H_plus_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_H_xeq_H_minus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_H_minus_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_r_times_H_minus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_r_times_H_minus_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_H_xeq_c_times_H_minus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_c_times_H_minus_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_H_xeq_pH_plus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_pH_plus_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_r_times_pH_plus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_r_times_pH_plus_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_H_xeq_c_times_pH_plus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_c_times_pH_plus_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_H_xeq_pH_minus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_pH_minus_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_r_times_pH_minus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_r_times_pH_minus_H(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_H_xeq_c_times_pH_minus_H (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_c_times_pH_minus_H(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_H_xeq_pH_plus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_pH_plus_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_r_times_pH_plus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_r_times_pH_plus_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_H_xeq_c_times_pH_plus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_c_times_pH_plus_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_H_xeq_pH_minus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_pH_minus_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_H_xeq_r_times_pH_minus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_r_times_pH_minus_pH(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_H_xeq_c_times_pH_minus_pH (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_H_xeq_c_times_pH_minus_pH(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* ---- ewise_d: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1335 (constant multiples of a field) */
/* replaces QLA_FN_D_veq_c_times_D (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_D_veq_c_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_veq_c_times_pD (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_D_veq_c_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_veq_C_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veq_C_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_veq_C_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veq_C_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_veq_pC_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veq_pC_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_veq_pC_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veq_pC_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_veq_Ca_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veq_Ca_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_veq_Ca_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veq_Ca_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_veq_pCa_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veq_pCa_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_veq_pCa_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veq_pCa_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_veq_R_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veq_R_times_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_veq_R_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veq_R_times_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_veq_pR_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veq_pR_times_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_veq_pR_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veq_pR_times_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_veq_conj_D (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_veq_conj_D(int nc, void * r, void * a, int n);
/* replaces QLA_FN_D_veq_conj_pD (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_veq_conj_pD(int nc, void * r, void * a, int n);
/* replaces QLA_FN_D_veq_i_D (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_veq_i_D(int nc, void * r, void * a, int n);
/* replaces QLA_FN_D_veq_i_pD (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_veq_i_pD(int nc, void * r, void * a, int n);
/* replaces QLA_FN_D_vpeq_c_times_D (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_D_vpeq_c_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_vpeq_c_times_pD (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_D_vpeq_c_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_vpeq_C_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vpeq_C_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_vpeq_C_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vpeq_C_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_vpeq_pC_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vpeq_pC_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_vpeq_pC_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vpeq_pC_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_vpeq_Ca_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vpeq_Ca_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_vpeq_Ca_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vpeq_Ca_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_vpeq_pCa_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vpeq_pCa_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_vpeq_pCa_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vpeq_pCa_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_vpeq_R_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vpeq_R_times_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_vpeq_R_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vpeq_R_times_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_vpeq_pR_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vpeq_pR_times_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_vpeq_pR_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vpeq_pR_times_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_vpeq_conj_D (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_vpeq_conj_D(int nc, void * r, void * a, int n);
/* replaces QLA_FN_D_vpeq_conj_pD (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_vpeq_conj_pD(int nc, void * r, void * a, int n);
/* replaces QLA_FN_D_vpeq_i_D (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_vpeq_i_D(int nc, void * r, void * a, int n);
/* replaces QLA_FN_D_vpeq_i_pD (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_vpeq_i_pD(int nc, void * r, void * a, int n);
/* replaces QLA_FN_D_vmeq_c_times_D (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_D_vmeq_c_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_vmeq_c_times_pD (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_D_vmeq_c_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_vmeq_C_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vmeq_C_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_vmeq_C_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vmeq_C_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_vmeq_pC_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vmeq_pC_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_vmeq_pC_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vmeq_pC_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_vmeq_Ca_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vmeq_Ca_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_vmeq_Ca_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vmeq_Ca_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_vmeq_pCa_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vmeq_pCa_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_vmeq_pCa_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vmeq_pCa_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_vmeq_R_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vmeq_R_times_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_vmeq_R_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vmeq_R_times_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_vmeq_pR_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vmeq_pR_times_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_vmeq_pR_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_vmeq_pR_times_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_vmeq_conj_D (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_vmeq_conj_D(int nc, void * r, void * a, int n);
/* replaces QLA_FN_D_vmeq_conj_pD (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_vmeq_conj_pD(int nc, void * r, void * a, int n);
/* replaces QLA_FN_D_vmeq_i_D (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_vmeq_i_D(int nc, void * r, void * a, int n);
/* replaces QLA_FN_D_vmeq_i_pD (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_vmeq_i_pD(int nc, void * r, void * a, int n);
/* replaces QLA_FN_D_veqm_c_times_D (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_D_veqm_c_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_veqm_c_times_pD (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_D_veqm_c_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_veqm_C_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veqm_C_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_veqm_C_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veqm_C_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_veqm_pC_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veqm_pC_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_veqm_pC_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veqm_pC_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_veqm_Ca_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veqm_Ca_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_veqm_Ca_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veqm_Ca_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_veqm_pCa_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veqm_pCa_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_veqm_pCa_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veqm_pCa_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_veqm_R_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veqm_R_times_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_veqm_R_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veqm_R_times_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_D_veqm_pR_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veqm_pR_times_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_veqm_pR_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_veqm_pR_times_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_D_veqm_conj_D (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_veqm_conj_D(int nc, void * r, void * a, int n);
/* replaces QLA_FN_D_veqm_conj_pD (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_veqm_conj_pD(int nc, void * r, void * a, int n);
/* replaces QLA_FN_D_veqm_i_D (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_veqm_i_D(int nc, void * r, void * a, int n);
/* replaces QLA_FN_D_veqm_i_pD (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_veqm_i_pD(int nc, void * r, void * a, int n);
/* replaces QLA_FN_D_veq_D_plus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_D_plus_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_veq_r_times_D_plus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_r_times_D_plus_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_D_veq_c_times_D_plus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_c_times_D_plus_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_D_veq_D_minus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_D_minus_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_veq_r_times_D_minus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_r_times_D_minus_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_D_veq_c_times_D_minus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_c_times_D_minus_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_D_veq_D_plus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_D_plus_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_veq_r_times_D_plus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_r_times_D_plus_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_D_veq_c_times_D_plus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_c_times_D_plus_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_D_veq_D_minus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_D_minus_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_veq_r_times_D_minus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_r_times_D_minus_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_D_veq_c_times_D_minus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_c_times_D_minus_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_D_veq_pD_plus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_pD_plus_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_veq_r_times_pD_plus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_r_times_pD_plus_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_D_veq_c_times_pD_plus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_c_times_pD_plus_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_D_veq_pD_minus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_pD_minus_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_veq_r_times_pD_minus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_r_times_pD_minus_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_D_veq_c_times_pD_minus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_c_times_pD_minus_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_D_veq_pD_plus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_pD_plus_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_veq_r_times_pD_plus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_r_times_pD_plus_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_D_veq_c_times_pD_plus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_c_times_pD_plus_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_D_veq_pD_minus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_pD_minus_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_D_veq_r_times_pD_minus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_r_times_pD_minus_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_D_veq_c_times_pD_minus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_veq_c_times_pD_minus_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_D_xeq_c_times_D (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_D_xeq_c_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_c_times_pD (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_D_xeq_c_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_C_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeq_C_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_C_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeq_C_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_pC_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeq_pC_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_pC_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeq_pC_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_Ca_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeq_Ca_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_Ca_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeq_Ca_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_pCa_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeq_pCa_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_pCa_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeq_pCa_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_R_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeq_R_times_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_R_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeq_R_times_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_pR_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeq_pR_times_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_pR_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeq_pR_times_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_conj_D (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_xeq_conj_D(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_D_xeq_conj_pD (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_xeq_conj_pD(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_D_xeq_i_D (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_xeq_i_D(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_D_xeq_i_pD (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_xeq_i_pD(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_D_xpeq_c_times_D (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_D_xpeq_c_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xpeq_c_times_pD (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_D_xpeq_c_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xpeq_C_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xpeq_C_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xpeq_C_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xpeq_C_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xpeq_pC_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xpeq_pC_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xpeq_pC_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xpeq_pC_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xpeq_Ca_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xpeq_Ca_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xpeq_Ca_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xpeq_Ca_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xpeq_pCa_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xpeq_pCa_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xpeq_pCa_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xpeq_pCa_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xpeq_R_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xpeq_R_times_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xpeq_R_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xpeq_R_times_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xpeq_pR_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xpeq_pR_times_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xpeq_pR_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xpeq_pR_times_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xpeq_conj_D (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_xpeq_conj_D(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_D_xpeq_conj_pD (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_xpeq_conj_pD(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_D_xpeq_i_D (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_xpeq_i_D(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_D_xpeq_i_pD (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_xpeq_i_pD(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_D_xmeq_c_times_D (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_D_xmeq_c_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xmeq_c_times_pD (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_D_xmeq_c_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xmeq_C_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xmeq_C_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xmeq_C_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xmeq_C_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xmeq_pC_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xmeq_pC_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xmeq_pC_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xmeq_pC_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xmeq_Ca_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xmeq_Ca_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xmeq_Ca_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xmeq_Ca_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xmeq_pCa_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xmeq_pCa_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xmeq_pCa_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xmeq_pCa_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xmeq_R_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xmeq_R_times_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xmeq_R_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xmeq_R_times_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xmeq_pR_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xmeq_pR_times_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xmeq_pR_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xmeq_pR_times_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xmeq_conj_D (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_xmeq_conj_D(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_D_xmeq_conj_pD (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_xmeq_conj_pD(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_D_xmeq_i_D (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_xmeq_i_D(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_D_xmeq_i_pD (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_xmeq_i_pD(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_D_xeqm_c_times_D (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_D_xeqm_c_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeqm_c_times_pD (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_D_xeqm_c_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeqm_C_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeqm_C_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeqm_C_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeqm_C_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeqm_pC_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeqm_pC_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeqm_pC_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeqm_pC_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeqm_Ca_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeqm_Ca_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeqm_Ca_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeqm_Ca_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeqm_pCa_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeqm_pCa_times_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeqm_pCa_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeqm_pCa_times_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeqm_R_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeqm_R_times_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeqm_R_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeqm_R_times_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeqm_pR_times_D (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeqm_pR_times_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeqm_pR_times_pD (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_D_xeqm_pR_times_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeqm_conj_D (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_xeqm_conj_D(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_D_xeqm_conj_pD (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_xeqm_conj_pD(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_D_xeqm_i_D (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_xeqm_i_D(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_D_xeqm_i_pD (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_D_xeqm_i_pD(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_D_xeq_D_plus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_D_plus_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_r_times_D_plus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_r_times_D_plus_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_D_xeq_c_times_D_plus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_c_times_D_plus_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_D_xeq_D_minus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_D_minus_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_r_times_D_minus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_r_times_D_minus_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_D_xeq_c_times_D_minus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_c_times_D_minus_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_D_xeq_D_plus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_D_plus_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_r_times_D_plus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_r_times_D_plus_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_D_xeq_c_times_D_plus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_c_times_D_plus_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_D_xeq_D_minus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_D_minus_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_r_times_D_minus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_r_times_D_minus_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_D_xeq_c_times_D_minus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_c_times_D_minus_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_D_xeq_pD_plus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_pD_plus_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_r_times_pD_plus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_r_times_pD_plus_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_D_xeq_c_times_pD_plus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_c_times_pD_plus_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_D_xeq_pD_minus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_pD_minus_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_r_times_pD_minus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_r_times_pD_minus_D(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_D_xeq_c_times_pD_minus_D (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_c_times_pD_minus_D(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_D_xeq_pD_plus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_pD_plus_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_r_times_pD_plus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_r_times_pD_plus_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_D_xeq_c_times_pD_plus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_c_times_pD_plus_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_D_xeq_pD_minus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_pD_minus_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_D_xeq_r_times_pD_minus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_r_times_pD_minus_pD(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_D_xeq_c_times_pD_minus_pD (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_D_xeq_c_times_pD_minus_pD(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* ---- ewise_m: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1335 (constant multiples of a field) */
/* replaces QLA_FN_M_veq_c_times_M (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_veq_c_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veq_c_times_pM (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_veq_c_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veq_c_times_Ma (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_veq_c_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veq_r_times_Ma (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_veq_r_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veq_c_times_pMa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_veq_c_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veq_r_times_pMa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_veq_r_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veq_C_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_C_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veq_C_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_C_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veq_C_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_C_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veq_C_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_C_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veq_pC_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_pC_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veq_pC_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_pC_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veq_pC_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_pC_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veq_pC_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_pC_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veq_Ca_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_Ca_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veq_Ca_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_Ca_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veq_Ca_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_Ca_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veq_Ca_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_Ca_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veq_pCa_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_pCa_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veq_pCa_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_pCa_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veq_pCa_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_pCa_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veq_pCa_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_pCa_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veq_R_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_R_times_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veq_R_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_R_times_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veq_R_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_R_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veq_R_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_R_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veq_pR_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_pR_times_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veq_pR_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_pR_times_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veq_pR_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_pR_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veq_pR_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veq_pR_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veq_conj_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_veq_conj_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_conj_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_veq_conj_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_i_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_veq_i_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_i_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_veq_i_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_Ma (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_veq_Ma(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_pMa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_veq_pMa(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_transpose_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_veq_transpose_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_transpose_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_veq_transpose_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_vpeq_c_times_M (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_vpeq_c_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vpeq_c_times_pM (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_vpeq_c_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vpeq_c_times_Ma (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_vpeq_c_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vpeq_r_times_Ma (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_vpeq_r_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vpeq_c_times_pMa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_vpeq_c_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vpeq_r_times_pMa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_vpeq_r_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vpeq_C_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_C_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vpeq_C_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_C_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vpeq_C_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_C_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vpeq_C_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_C_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vpeq_pC_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_pC_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_pC_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_pC_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_pC_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_pC_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_pC_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_pC_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_Ca_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_Ca_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vpeq_Ca_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_Ca_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vpeq_Ca_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_Ca_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vpeq_Ca_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_Ca_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vpeq_pCa_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_pCa_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_pCa_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_pCa_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_pCa_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_pCa_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_pCa_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_pCa_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_R_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_R_times_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vpeq_R_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_R_times_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vpeq_R_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_R_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vpeq_R_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_R_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vpeq_pR_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_pR_times_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_pR_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_pR_times_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_pR_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_pR_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_pR_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vpeq_pR_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_conj_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_vpeq_conj_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_vpeq_conj_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_vpeq_conj_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_vpeq_i_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_vpeq_i_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_vpeq_i_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_vpeq_i_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_vpeq_Ma (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_vpeq_Ma(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_vpeq_pMa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_vpeq_pMa(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_vpeq_transpose_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_vpeq_transpose_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_vpeq_transpose_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_vpeq_transpose_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_vmeq_c_times_M (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_vmeq_c_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vmeq_c_times_pM (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_vmeq_c_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vmeq_c_times_Ma (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_vmeq_c_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vmeq_r_times_Ma (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_vmeq_r_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vmeq_c_times_pMa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_vmeq_c_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vmeq_r_times_pMa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_vmeq_r_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vmeq_C_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_C_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vmeq_C_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_C_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vmeq_C_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_C_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vmeq_C_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_C_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vmeq_pC_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_pC_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_pC_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_pC_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_pC_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_pC_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_pC_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_pC_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_Ca_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_Ca_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vmeq_Ca_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_Ca_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vmeq_Ca_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_Ca_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vmeq_Ca_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_Ca_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vmeq_pCa_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_pCa_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_pCa_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_pCa_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_pCa_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_pCa_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_pCa_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_pCa_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_R_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_R_times_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vmeq_R_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_R_times_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vmeq_R_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_R_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vmeq_R_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_R_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_vmeq_pR_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_pR_times_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_pR_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_pR_times_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_pR_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_pR_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_pR_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_vmeq_pR_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_conj_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_vmeq_conj_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_vmeq_conj_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_vmeq_conj_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_vmeq_i_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_vmeq_i_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_vmeq_i_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_vmeq_i_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_vmeq_Ma (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_vmeq_Ma(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_vmeq_pMa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_vmeq_pMa(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_vmeq_transpose_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_vmeq_transpose_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_vmeq_transpose_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_vmeq_transpose_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veqm_c_times_M (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_veqm_c_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veqm_c_times_pM (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_veqm_c_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veqm_c_times_Ma (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_veqm_c_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veqm_r_times_Ma (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_veqm_r_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veqm_c_times_pMa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_veqm_c_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veqm_r_times_pMa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_veqm_r_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veqm_C_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_C_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veqm_C_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_C_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veqm_C_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_C_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veqm_C_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_C_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veqm_pC_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_pC_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veqm_pC_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_pC_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veqm_pC_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_pC_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veqm_pC_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_pC_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veqm_Ca_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_Ca_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veqm_Ca_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_Ca_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veqm_Ca_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_Ca_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veqm_Ca_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_Ca_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veqm_pCa_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_pCa_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veqm_pCa_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_pCa_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veqm_pCa_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_pCa_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veqm_pCa_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_pCa_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veqm_R_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_R_times_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veqm_R_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_R_times_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veqm_R_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_R_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veqm_R_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_R_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_M_veqm_pR_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_pR_times_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veqm_pR_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_pR_times_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veqm_pR_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_pR_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veqm_pR_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_veqm_pR_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_M_veqm_conj_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_veqm_conj_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veqm_conj_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_veqm_conj_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veqm_i_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_veqm_i_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veqm_i_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_veqm_i_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veqm_Ma (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_veqm_Ma(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veqm_pMa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_veqm_pMa(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veqm_transpose_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_veqm_transpose_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veqm_transpose_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_veqm_transpose_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_M_plus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_M_plus_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_r_times_M_plus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_r_times_M_plus_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_M_veq_c_times_M_plus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_c_times_M_plus_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_M_veq_M_minus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_M_minus_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_r_times_M_minus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_r_times_M_minus_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_M_veq_c_times_M_minus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_c_times_M_minus_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_M_veq_M_plus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_M_plus_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_r_times_M_plus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_r_times_M_plus_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_M_veq_c_times_M_plus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_c_times_M_plus_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_M_veq_M_minus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_M_minus_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_r_times_M_minus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_r_times_M_minus_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_M_veq_c_times_M_minus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_c_times_M_minus_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_M_veq_pM_plus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_pM_plus_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_r_times_pM_plus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_r_times_pM_plus_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_M_veq_c_times_pM_plus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_c_times_pM_plus_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_M_veq_pM_minus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_pM_minus_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_r_times_pM_minus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_r_times_pM_minus_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_M_veq_c_times_pM_minus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_c_times_pM_minus_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_M_veq_pM_plus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_pM_plus_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_r_times_pM_plus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_r_times_pM_plus_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_M_veq_c_times_pM_plus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_c_times_pM_plus_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_M_veq_pM_minus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_pM_minus_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_r_times_pM_minus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_r_times_pM_minus_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_M_veq_c_times_pM_minus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_veq_c_times_pM_minus_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_M_xeq_c_times_M (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xeq_c_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_c_times_pM (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xeq_c_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_c_times_Ma (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xeq_c_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_r_times_Ma (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xeq_r_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_c_times_pMa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xeq_c_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_r_times_pMa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xeq_r_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_C_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_C_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_C_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_C_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_C_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_C_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_C_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_C_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pC_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_pC_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pC_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_pC_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pC_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_pC_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pC_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_pC_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_Ca_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_Ca_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_Ca_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_Ca_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_Ca_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_Ca_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_Ca_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_Ca_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pCa_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_pCa_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pCa_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_pCa_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pCa_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_pCa_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pCa_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_pCa_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_R_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_R_times_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_R_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_R_times_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_R_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_R_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_R_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_R_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pR_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_pR_times_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pR_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_pR_times_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pR_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_pR_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pR_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeq_pR_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_conj_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xeq_conj_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_conj_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xeq_conj_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_i_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xeq_i_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_i_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xeq_i_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_Ma (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xeq_Ma(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_pMa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xeq_pMa(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_transpose_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xeq_transpose_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_transpose_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xeq_transpose_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xpeq_c_times_M (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xpeq_c_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_c_times_pM (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xpeq_c_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_c_times_Ma (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xpeq_c_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_r_times_Ma (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xpeq_r_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_c_times_pMa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xpeq_c_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_r_times_pMa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xpeq_r_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_C_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_C_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_C_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_C_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_C_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_C_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_C_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_C_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_pC_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_pC_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_pC_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_pC_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_pC_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_pC_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_pC_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_pC_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_Ca_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_Ca_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_Ca_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_Ca_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_Ca_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_Ca_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_Ca_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_Ca_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_pCa_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_pCa_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_pCa_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_pCa_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_pCa_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_pCa_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_pCa_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_pCa_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_R_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_R_times_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_R_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_R_times_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_R_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_R_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_R_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_R_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_pR_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_pR_times_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_pR_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_pR_times_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_pR_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_pR_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_pR_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xpeq_pR_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_conj_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xpeq_conj_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xpeq_conj_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xpeq_conj_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xpeq_i_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xpeq_i_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xpeq_i_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xpeq_i_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xpeq_Ma (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xpeq_Ma(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xpeq_pMa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xpeq_pMa(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xpeq_transpose_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xpeq_transpose_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xpeq_transpose_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xpeq_transpose_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xmeq_c_times_M (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xmeq_c_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_c_times_pM (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xmeq_c_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_c_times_Ma (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xmeq_c_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_r_times_Ma (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xmeq_r_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_c_times_pMa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xmeq_c_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_r_times_pMa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xmeq_r_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_C_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_C_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_C_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_C_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_C_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_C_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_C_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_C_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_pC_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_pC_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_pC_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_pC_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_pC_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_pC_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_pC_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_pC_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_Ca_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_Ca_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_Ca_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_Ca_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_Ca_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_Ca_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_Ca_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_Ca_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_pCa_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_pCa_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_pCa_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_pCa_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_pCa_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_pCa_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_pCa_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_pCa_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_R_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_R_times_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_R_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_R_times_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_R_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_R_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_R_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_R_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_pR_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_pR_times_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_pR_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_pR_times_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_pR_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_pR_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_pR_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xmeq_pR_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_conj_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xmeq_conj_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xmeq_conj_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xmeq_conj_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xmeq_i_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xmeq_i_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xmeq_i_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xmeq_i_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xmeq_Ma (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xmeq_Ma(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xmeq_pMa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xmeq_pMa(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xmeq_transpose_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xmeq_transpose_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xmeq_transpose_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xmeq_transpose_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeqm_c_times_M (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xeqm_c_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_c_times_pM (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xeqm_c_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_c_times_Ma (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xeqm_c_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_r_times_Ma (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xeqm_r_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_c_times_pMa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xeqm_c_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_r_times_pMa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_M_xeqm_r_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_C_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_C_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_C_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_C_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_C_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_C_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_C_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_C_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_pC_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_pC_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_pC_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_pC_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_pC_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_pC_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_pC_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_pC_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_Ca_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_Ca_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_Ca_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_Ca_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_Ca_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_Ca_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_Ca_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_Ca_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_pCa_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_pCa_times_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_pCa_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_pCa_times_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_pCa_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_pCa_times_Ma(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_pCa_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_pCa_times_pMa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_R_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_R_times_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_R_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_R_times_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_R_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_R_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_R_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_R_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_pR_times_M (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_pR_times_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_pR_times_pM (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_pR_times_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_pR_times_Ma (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_pR_times_Ma(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_pR_times_pMa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_M_xeqm_pR_times_pMa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_conj_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xeqm_conj_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeqm_conj_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xeqm_conj_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeqm_i_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xeqm_i_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeqm_i_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xeqm_i_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeqm_Ma (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xeqm_Ma(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeqm_pMa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xeqm_pMa(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeqm_transpose_M (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xeqm_transpose_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeqm_transpose_pM (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_M_xeqm_transpose_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_M_plus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_M_plus_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_r_times_M_plus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_r_times_M_plus_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_M_xeq_c_times_M_plus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_c_times_M_plus_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_M_xeq_M_minus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_M_minus_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_r_times_M_minus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_r_times_M_minus_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_M_xeq_c_times_M_minus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_c_times_M_minus_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_M_xeq_M_plus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_M_plus_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_r_times_M_plus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_r_times_M_plus_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_M_xeq_c_times_M_plus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_c_times_M_plus_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_M_xeq_M_minus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_M_minus_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_r_times_M_minus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_r_times_M_minus_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_M_xeq_c_times_M_minus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_c_times_M_minus_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_M_xeq_pM_plus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_pM_plus_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_r_times_pM_plus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_r_times_pM_plus_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_M_xeq_c_times_pM_plus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_c_times_pM_plus_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_M_xeq_pM_minus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_pM_minus_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_r_times_pM_minus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_r_times_pM_minus_M(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_M_xeq_c_times_pM_minus_M (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_c_times_pM_minus_M(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_M_xeq_pM_plus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_pM_plus_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_r_times_pM_plus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_r_times_pM_plus_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_M_xeq_c_times_pM_plus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_c_times_pM_plus_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_M_xeq_pM_minus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_pM_minus_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_r_times_pM_minus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_r_times_pM_minus_pM(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_M_xeq_c_times_pM_minus_pM (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_M_xeq_c_times_pM_minus_pM(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* ---- ewise_p: replaces the FN functions emitted by lib/perl/build_qla.pl:1256-1335 (constant multiples of a field) */
/* replaces QLA_FN_P_veq_c_times_P (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_veq_c_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veq_r_times_P (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_veq_r_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veq_c_times_pP (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_veq_c_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veq_r_times_pP (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_veq_r_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veq_c_times_Pa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_veq_c_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veq_r_times_Pa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_veq_r_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veq_c_times_pPa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_veq_c_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veq_r_times_pPa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_veq_r_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veq_C_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_C_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veq_C_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_C_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veq_C_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_C_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veq_C_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_C_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veq_pC_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_pC_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veq_pC_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_pC_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veq_pC_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_pC_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veq_pC_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_pC_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veq_Ca_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_Ca_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veq_Ca_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_Ca_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veq_Ca_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_Ca_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veq_Ca_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_Ca_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veq_pCa_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_pCa_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veq_pCa_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_pCa_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veq_pCa_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_pCa_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veq_pCa_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_pCa_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veq_R_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_R_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veq_R_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_R_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veq_R_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_R_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veq_R_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_R_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veq_pR_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_pR_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veq_pR_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_pR_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veq_pR_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_pR_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veq_pR_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veq_pR_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veq_conj_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_veq_conj_P(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_veq_conj_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_veq_conj_pP(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_veq_i_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_veq_i_P(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_veq_i_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_veq_i_pP(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_veq_Pa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_veq_Pa(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_veq_pPa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_veq_pPa(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_veq_transpose_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_veq_transpose_P(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_veq_transpose_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_veq_transpose_pP(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_veq_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_veq_P(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_veq_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_veq_pP(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_vpeq_c_times_P (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_vpeq_c_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vpeq_r_times_P (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_vpeq_r_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vpeq_c_times_pP (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_vpeq_c_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vpeq_r_times_pP (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_vpeq_r_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vpeq_c_times_Pa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_vpeq_c_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vpeq_r_times_Pa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_vpeq_r_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vpeq_c_times_pPa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_vpeq_c_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vpeq_r_times_pPa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_vpeq_r_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vpeq_C_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_C_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vpeq_C_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_C_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vpeq_C_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_C_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vpeq_C_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_C_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pC_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_pC_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pC_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_pC_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pC_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_pC_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pC_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_pC_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_Ca_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_Ca_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vpeq_Ca_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_Ca_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vpeq_Ca_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_Ca_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vpeq_Ca_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_Ca_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pCa_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_pCa_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pCa_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_pCa_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pCa_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_pCa_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pCa_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_pCa_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_R_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_R_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vpeq_R_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_R_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vpeq_R_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_R_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vpeq_R_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_R_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pR_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_pR_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pR_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_pR_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pR_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_pR_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pR_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vpeq_pR_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_conj_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_vpeq_conj_P(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_vpeq_conj_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_vpeq_conj_pP(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_vpeq_i_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_vpeq_i_P(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_vpeq_i_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_vpeq_i_pP(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_vpeq_Pa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_vpeq_Pa(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_vpeq_pPa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_vpeq_pPa(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_vpeq_transpose_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_vpeq_transpose_P(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_vpeq_transpose_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_vpeq_transpose_pP(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_vpeq_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_vpeq_P(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_vpeq_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_vpeq_pP(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_vmeq_c_times_P (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_vmeq_c_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vmeq_r_times_P (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_vmeq_r_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vmeq_c_times_pP (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_vmeq_c_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vmeq_r_times_pP (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_vmeq_r_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vmeq_c_times_Pa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_vmeq_c_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vmeq_r_times_Pa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_vmeq_r_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vmeq_c_times_pPa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_vmeq_c_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vmeq_r_times_pPa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_vmeq_r_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vmeq_C_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_C_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vmeq_C_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_C_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vmeq_C_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_C_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vmeq_C_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_C_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pC_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_pC_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pC_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_pC_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pC_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_pC_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pC_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_pC_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_Ca_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_Ca_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vmeq_Ca_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_Ca_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vmeq_Ca_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_Ca_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vmeq_Ca_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_Ca_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pCa_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_pCa_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pCa_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_pCa_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pCa_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_pCa_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pCa_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_pCa_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_R_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_R_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vmeq_R_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_R_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vmeq_R_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_R_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vmeq_R_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_R_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pR_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_pR_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pR_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_pR_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pR_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_pR_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pR_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_vmeq_pR_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_conj_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_vmeq_conj_P(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_vmeq_conj_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_vmeq_conj_pP(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_vmeq_i_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_vmeq_i_P(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_vmeq_i_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_vmeq_i_pP(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_vmeq_Pa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_vmeq_Pa(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_vmeq_pPa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_vmeq_pPa(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_vmeq_transpose_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_vmeq_transpose_P(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_vmeq_transpose_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_vmeq_transpose_pP(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_vmeq_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_vmeq_P(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_vmeq_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_vmeq_pP(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_veqm_c_times_P (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_veqm_c_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veqm_r_times_P (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_veqm_r_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veqm_c_times_pP (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_veqm_c_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veqm_r_times_pP (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_veqm_r_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veqm_c_times_Pa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_veqm_c_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veqm_r_times_Pa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_veqm_r_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veqm_c_times_pPa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_veqm_c_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veqm_r_times_pPa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_veqm_r_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veqm_C_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_C_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veqm_C_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_C_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veqm_C_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_C_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veqm_C_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_C_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veqm_pC_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_pC_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pC_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_pC_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pC_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_pC_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pC_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_pC_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veqm_Ca_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_Ca_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veqm_Ca_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_Ca_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veqm_Ca_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_Ca_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veqm_Ca_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_Ca_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veqm_pCa_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_pCa_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pCa_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_pCa_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pCa_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_pCa_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pCa_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_pCa_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veqm_R_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_R_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veqm_R_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_R_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veqm_R_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_R_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veqm_R_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_R_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int n);
/* replaces QLA_FN_P_veqm_pR_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_pR_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pR_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_pR_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pR_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_pR_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pR_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_veqm_pR_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int n);
/* replaces QLA_FN_P_veqm_conj_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_veqm_conj_P(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_veqm_conj_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_veqm_conj_pP(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_veqm_i_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_veqm_i_P(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_veqm_i_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_veqm_i_pP(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_veqm_Pa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_veqm_Pa(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_veqm_pPa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_veqm_pPa(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_veqm_transpose_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_veqm_transpose_P(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_veqm_transpose_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_veqm_transpose_pP(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_veqm_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_veqm_P(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_veqm_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_veqm_pP(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_veq_P_plus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_P_plus_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_r_times_P_plus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_r_times_P_plus_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_P_veq_c_times_P_plus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_c_times_P_plus_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_P_veq_P_minus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_P_minus_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_r_times_P_minus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_r_times_P_minus_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_P_veq_c_times_P_minus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_c_times_P_minus_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_P_veq_P_plus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_P_plus_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_r_times_P_plus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_r_times_P_plus_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_P_veq_c_times_P_plus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_c_times_P_plus_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_P_veq_P_minus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_P_minus_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_r_times_P_minus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_r_times_P_minus_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_P_veq_c_times_P_minus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_c_times_P_minus_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_P_veq_pP_plus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_pP_plus_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_r_times_pP_plus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_r_times_pP_plus_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_P_veq_c_times_pP_plus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_c_times_pP_plus_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_P_veq_pP_minus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_pP_minus_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_r_times_pP_minus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_r_times_pP_minus_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_P_veq_c_times_pP_minus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_c_times_pP_minus_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_P_veq_pP_plus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_pP_plus_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_r_times_pP_plus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_r_times_pP_plus_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_P_veq_c_times_pP_plus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_c_times_pP_plus_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_P_veq_pP_minus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_pP_minus_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_r_times_pP_minus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_r_times_pP_minus_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_P_veq_c_times_pP_minus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_veq_c_times_pP_minus_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int n);
/* replaces QLA_FN_P_xeq_c_times_P (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xeq_c_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_r_times_P (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xeq_r_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_c_times_pP (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xeq_c_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_r_times_pP (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xeq_r_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_c_times_Pa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xeq_c_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_r_times_Pa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xeq_r_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_c_times_pPa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xeq_c_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_r_times_pPa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xeq_r_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_C_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_C_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_C_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_C_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_C_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_C_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_C_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_C_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pC_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_pC_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pC_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_pC_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pC_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_pC_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pC_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_pC_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_Ca_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_Ca_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_Ca_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_Ca_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_Ca_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_Ca_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_Ca_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_Ca_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pCa_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_pCa_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pCa_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_pCa_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pCa_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_pCa_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pCa_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_pCa_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_R_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_R_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_R_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_R_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_R_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_R_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_R_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_R_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pR_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_pR_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pR_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_pR_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pR_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_pR_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pR_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeq_pR_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_conj_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xeq_conj_P(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xeq_conj_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xeq_conj_pP(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xeq_i_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xeq_i_P(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xeq_i_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xeq_i_pP(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xeq_Pa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xeq_Pa(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xeq_pPa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xeq_pPa(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xeq_transpose_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xeq_transpose_P(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xeq_transpose_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xeq_transpose_pP(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xeq_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xeq_P(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xeq_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xeq_pP(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xpeq_c_times_P (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xpeq_c_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_r_times_P (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xpeq_r_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_c_times_pP (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xpeq_c_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_r_times_pP (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xpeq_r_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_c_times_Pa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xpeq_c_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_r_times_Pa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xpeq_r_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_c_times_pPa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xpeq_c_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_r_times_pPa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xpeq_r_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_C_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_C_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_C_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_C_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_C_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_C_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_C_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_C_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pC_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_pC_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pC_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_pC_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pC_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_pC_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pC_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_pC_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_Ca_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_Ca_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_Ca_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_Ca_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_Ca_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_Ca_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_Ca_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_Ca_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pCa_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_pCa_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pCa_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_pCa_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pCa_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_pCa_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pCa_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_pCa_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_R_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_R_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_R_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_R_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_R_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_R_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_R_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_R_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pR_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_pR_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pR_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_pR_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pR_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_pR_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pR_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xpeq_pR_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_conj_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xpeq_conj_P(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xpeq_conj_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xpeq_conj_pP(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xpeq_i_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xpeq_i_P(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xpeq_i_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xpeq_i_pP(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xpeq_Pa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xpeq_Pa(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xpeq_pPa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xpeq_pPa(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xpeq_transpose_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xpeq_transpose_P(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xpeq_transpose_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xpeq_transpose_pP(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xpeq_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xpeq_P(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xpeq_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xpeq_pP(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xmeq_c_times_P (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xmeq_c_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_r_times_P (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xmeq_r_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_c_times_pP (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xmeq_c_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_r_times_pP (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xmeq_r_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_c_times_Pa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xmeq_c_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_r_times_Pa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xmeq_r_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_c_times_pPa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xmeq_c_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_r_times_pPa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xmeq_r_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_C_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_C_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_C_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_C_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_C_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_C_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_C_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_C_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pC_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_pC_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pC_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_pC_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pC_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_pC_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pC_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_pC_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_Ca_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_Ca_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_Ca_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_Ca_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_Ca_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_Ca_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_Ca_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_Ca_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pCa_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_pCa_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pCa_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_pCa_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pCa_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_pCa_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pCa_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_pCa_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_R_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_R_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_R_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_R_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_R_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_R_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_R_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_R_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pR_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_pR_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pR_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_pR_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pR_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_pR_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pR_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xmeq_pR_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_conj_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xmeq_conj_P(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xmeq_conj_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xmeq_conj_pP(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xmeq_i_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xmeq_i_P(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xmeq_i_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xmeq_i_pP(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xmeq_Pa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xmeq_Pa(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xmeq_pPa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xmeq_pPa(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xmeq_transpose_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xmeq_transpose_P(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xmeq_transpose_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xmeq_transpose_pP(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xmeq_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xmeq_P(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xmeq_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xmeq_pP(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xeqm_c_times_P (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xeqm_c_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_r_times_P (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xeqm_r_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_c_times_pP (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xeqm_c_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_r_times_pP (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xeqm_r_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_c_times_Pa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xeqm_c_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_r_times_Pa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xeqm_r_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_c_times_pPa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xeqm_c_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_r_times_pPa (lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400) */
void QLA_FN_P_xeqm_r_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_C_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_C_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_C_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_C_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_C_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_C_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_C_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_C_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pC_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_pC_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pC_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_pC_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pC_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_pC_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pC_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_pC_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_Ca_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_Ca_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_Ca_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_Ca_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_Ca_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_Ca_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_Ca_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_Ca_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pCa_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_pCa_times_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pCa_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_pCa_times_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pCa_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_pCa_times_Pa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pCa_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_pCa_times_pPa(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_R_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_R_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_R_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_R_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_R_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_R_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_R_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_R_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pR_times_P (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_pR_times_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pR_times_pP (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_pR_times_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pR_times_Pa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_pR_times_Pa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pR_times_pPa (lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)) */
void QLA_FN_P_xeqm_pR_times_pPa(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_conj_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xeqm_conj_P(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xeqm_conj_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xeqm_conj_pP(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xeqm_i_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xeqm_i_P(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xeqm_i_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xeqm_i_pP(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xeqm_Pa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xeqm_Pa(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xeqm_pPa (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xeqm_pPa(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xeqm_transpose_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xeqm_transpose_P(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xeqm_transpose_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xeqm_transpose_pP(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xeqm_P (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xeqm_P(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xeqm_pP (lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)) */
void QLA_FN_P_xeqm_pP(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xeq_P_plus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_P_plus_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_r_times_P_plus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_r_times_P_plus_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_P_xeq_c_times_P_plus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_c_times_P_plus_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_P_xeq_P_minus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_P_minus_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_r_times_P_minus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_r_times_P_minus_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_P_xeq_c_times_P_minus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_c_times_P_minus_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_P_xeq_P_plus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_P_plus_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_r_times_P_plus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_r_times_P_plus_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_P_xeq_c_times_P_plus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_c_times_P_plus_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_P_xeq_P_minus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_P_minus_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_r_times_P_minus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_r_times_P_minus_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_P_xeq_c_times_P_minus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_c_times_P_minus_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_P_xeq_pP_plus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_pP_plus_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_r_times_pP_plus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_r_times_pP_plus_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_P_xeq_c_times_pP_plus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_c_times_pP_plus_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_P_xeq_pP_minus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_pP_minus_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_r_times_pP_minus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_r_times_pP_minus_P(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_P_xeq_c_times_pP_minus_P (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_c_times_pP_minus_P(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_P_xeq_pP_plus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_pP_plus_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_r_times_pP_plus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_r_times_pP_plus_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_P_xeq_c_times_pP_plus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_c_times_pP_plus_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_P_xeq_pP_minus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_pP_minus_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_r_times_pP_minus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_r_times_pP_minus_pP(int nc, void * r, QLA_F_Real *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* replaces QLA_FN_P_xeq_c_times_pP_minus_pP (lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)) */
void QLA_FN_P_xeq_c_times_pP_minus_pP(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, void * b, void * c, int * index, int n);
/* ---- ldot: replaces the FN functions emitted by lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms) */
/* replaces QLA_FN_C_veq_V_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_V_dot_V(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_re_V_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_re_V_dot_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_V_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_V_dot_pV(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_re_V_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_re_V_dot_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_pV_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_pV_dot_V(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_re_pV_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_re_pV_dot_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_pV_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_pV_dot_pV(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_re_pV_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_re_pV_dot_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_norm2_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_norm2_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_veq_norm2_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_norm2_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_C_vpeq_V_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_V_dot_V(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_re_V_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_re_V_dot_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_V_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_V_dot_pV(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_re_V_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_re_V_dot_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_pV_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_pV_dot_V(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_re_pV_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_re_pV_dot_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_pV_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_pV_dot_pV(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_re_pV_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_re_pV_dot_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_norm2_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_norm2_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_vpeq_norm2_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_norm2_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_C_vmeq_V_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_V_dot_V(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_re_V_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_re_V_dot_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_V_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_V_dot_pV(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_re_V_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_re_V_dot_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_pV_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_pV_dot_V(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_re_pV_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_re_pV_dot_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_pV_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_pV_dot_pV(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_re_pV_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_re_pV_dot_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_norm2_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_norm2_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_vmeq_norm2_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_norm2_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_C_veqm_V_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_V_dot_V(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_re_V_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_re_V_dot_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_V_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_V_dot_pV(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_re_V_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_re_V_dot_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_pV_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_pV_dot_V(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_re_pV_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_re_pV_dot_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_pV_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_pV_dot_pV(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_re_pV_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_re_pV_dot_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_norm2_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_norm2_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_veqm_norm2_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_norm2_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_C_xeq_V_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_V_dot_V(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_re_V_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_re_V_dot_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_V_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_V_dot_pV(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_re_V_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_re_V_dot_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_pV_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_pV_dot_V(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_re_pV_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_re_pV_dot_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_pV_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_pV_dot_pV(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_re_pV_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_re_pV_dot_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_norm2_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_norm2_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xeq_norm2_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_norm2_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_C_xpeq_V_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_V_dot_V(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_re_V_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_re_V_dot_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_V_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_V_dot_pV(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_re_V_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_re_V_dot_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_pV_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_pV_dot_V(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_re_pV_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_re_pV_dot_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_pV_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_pV_dot_pV(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_re_pV_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_re_pV_dot_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_norm2_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_norm2_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xpeq_norm2_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_norm2_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_C_xmeq_V_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_V_dot_V(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_re_V_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_re_V_dot_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_V_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_V_dot_pV(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_re_V_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_re_V_dot_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_pV_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_pV_dot_V(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_re_pV_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_re_pV_dot_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_pV_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_pV_dot_pV(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_re_pV_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_re_pV_dot_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_norm2_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_norm2_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xmeq_norm2_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_norm2_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_C_xeqm_V_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_V_dot_V(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_re_V_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_re_V_dot_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_V_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_V_dot_pV(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_re_V_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_re_V_dot_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_pV_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_pV_dot_V(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_re_pV_dot_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_re_pV_dot_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_pV_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_pV_dot_pV(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_re_pV_dot_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_re_pV_dot_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_norm2_V (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_norm2_V(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xeqm_norm2_pV (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_norm2_pV(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_C_veq_H_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_H_dot_H(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_re_H_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_re_H_dot_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_H_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_H_dot_pH(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_re_H_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_re_H_dot_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_pH_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_pH_dot_H(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_re_pH_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_re_pH_dot_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_pH_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_pH_dot_pH(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_re_pH_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_re_pH_dot_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_norm2_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_norm2_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_veq_norm2_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_norm2_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_C_vpeq_H_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_H_dot_H(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_re_H_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_re_H_dot_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_H_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_H_dot_pH(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_re_H_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_re_H_dot_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_pH_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_pH_dot_H(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_re_pH_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_re_pH_dot_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_pH_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_pH_dot_pH(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_re_pH_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_re_pH_dot_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_norm2_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_norm2_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_vpeq_norm2_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_norm2_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_C_vmeq_H_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_H_dot_H(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_re_H_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_re_H_dot_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_H_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_H_dot_pH(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_re_H_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_re_H_dot_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_pH_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_pH_dot_H(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_re_pH_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_re_pH_dot_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_pH_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_pH_dot_pH(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_re_pH_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_re_pH_dot_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_norm2_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_norm2_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_vmeq_norm2_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_norm2_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_C_veqm_H_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_H_dot_H(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_re_H_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_re_H_dot_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_H_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_H_dot_pH(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_re_H_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_re_H_dot_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_pH_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_pH_dot_H(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_re_pH_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_re_pH_dot_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_pH_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_pH_dot_pH(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_re_pH_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_re_pH_dot_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_norm2_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_norm2_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_veqm_norm2_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_norm2_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_C_xeq_H_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_H_dot_H(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_re_H_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_re_H_dot_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_H_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_H_dot_pH(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_re_H_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_re_H_dot_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_pH_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_pH_dot_H(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_re_pH_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_re_pH_dot_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_pH_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_pH_dot_pH(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_re_pH_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_re_pH_dot_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_norm2_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_norm2_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xeq_norm2_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_norm2_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_C_xpeq_H_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_H_dot_H(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_re_H_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_re_H_dot_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_H_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_H_dot_pH(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_re_H_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_re_H_dot_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_pH_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_pH_dot_H(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_re_pH_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_re_pH_dot_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_pH_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_pH_dot_pH(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_re_pH_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_re_pH_dot_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_norm2_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_norm2_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xpeq_norm2_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_norm2_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_C_xmeq_H_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_H_dot_H(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_re_H_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_re_H_dot_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_H_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_H_dot_pH(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_re_H_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_re_H_dot_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_pH_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_pH_dot_H(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_re_pH_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_re_pH_dot_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_pH_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_pH_dot_pH(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_re_pH_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_re_pH_dot_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_norm2_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_norm2_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xmeq_norm2_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_norm2_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_C_xeqm_H_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_H_dot_H(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_re_H_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_re_H_dot_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_H_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_H_dot_pH(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_re_H_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_re_H_dot_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_pH_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_pH_dot_H(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_re_pH_dot_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_re_pH_dot_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_pH_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_pH_dot_pH(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_re_pH_dot_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_re_pH_dot_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_norm2_H (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_norm2_H(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xeqm_norm2_pH (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_norm2_pH(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_C_veq_D_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_D_dot_D(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_re_D_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_re_D_dot_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_D_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_D_dot_pD(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_re_D_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_re_D_dot_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_pD_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_pD_dot_D(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_re_pD_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_re_pD_dot_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_pD_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_pD_dot_pD(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_re_pD_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_re_pD_dot_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_norm2_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_norm2_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_veq_norm2_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_norm2_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_C_vpeq_D_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_D_dot_D(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_re_D_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_re_D_dot_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_D_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_D_dot_pD(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_re_D_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_re_D_dot_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_pD_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_pD_dot_D(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_re_pD_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_re_pD_dot_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_pD_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_pD_dot_pD(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_re_pD_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_re_pD_dot_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_norm2_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_norm2_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_vpeq_norm2_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_norm2_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_C_vmeq_D_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_D_dot_D(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_re_D_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_re_D_dot_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_D_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_D_dot_pD(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_re_D_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_re_D_dot_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_pD_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_pD_dot_D(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_re_pD_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_re_pD_dot_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_pD_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_pD_dot_pD(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_re_pD_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_re_pD_dot_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_norm2_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_norm2_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_vmeq_norm2_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_norm2_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_C_veqm_D_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_D_dot_D(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_re_D_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_re_D_dot_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_D_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_D_dot_pD(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_re_D_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_re_D_dot_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_pD_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_pD_dot_D(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_re_pD_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_re_pD_dot_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_pD_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_pD_dot_pD(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_re_pD_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_re_pD_dot_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_norm2_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_norm2_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_veqm_norm2_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_norm2_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_C_xeq_D_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_D_dot_D(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_re_D_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_re_D_dot_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_D_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_D_dot_pD(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_re_D_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_re_D_dot_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_pD_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_pD_dot_D(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_re_pD_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_re_pD_dot_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_pD_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_pD_dot_pD(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_re_pD_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_re_pD_dot_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_norm2_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_norm2_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xeq_norm2_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_norm2_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_C_xpeq_D_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_D_dot_D(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_re_D_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_re_D_dot_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_D_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_D_dot_pD(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_re_D_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_re_D_dot_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_pD_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_pD_dot_D(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_re_pD_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_re_pD_dot_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_pD_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_pD_dot_pD(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_re_pD_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_re_pD_dot_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_norm2_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_norm2_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xpeq_norm2_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_norm2_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_C_xmeq_D_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_D_dot_D(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_re_D_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_re_D_dot_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_D_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_D_dot_pD(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_re_D_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_re_D_dot_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_pD_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_pD_dot_D(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_re_pD_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_re_pD_dot_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_pD_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_pD_dot_pD(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_re_pD_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_re_pD_dot_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_norm2_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_norm2_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xmeq_norm2_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_norm2_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_C_xeqm_D_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_D_dot_D(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_re_D_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_re_D_dot_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_D_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_D_dot_pD(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_re_D_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_re_D_dot_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_pD_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_pD_dot_D(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_re_pD_dot_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_re_pD_dot_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_pD_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_pD_dot_pD(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_re_pD_dot_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_re_pD_dot_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_norm2_D (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_norm2_D(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xeqm_norm2_pD (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_norm2_pD(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_C_veq_M_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_M_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_re_M_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_re_M_dot_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_M_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_M_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_re_M_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_re_M_dot_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_pM_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_pM_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_re_pM_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_re_pM_dot_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_pM_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_pM_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_re_pM_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_re_pM_dot_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_M_dot_Ma (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_M_dot_Ma(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_M_dot_pMa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_M_dot_pMa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_pM_dot_Ma (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_pM_dot_Ma(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_pM_dot_pMa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_pM_dot_pMa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_Ma_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_Ma_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_Ma_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_Ma_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_pMa_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_pMa_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_pMa_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_pMa_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_norm2_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_norm2_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_veq_norm2_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_norm2_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_C_vpeq_M_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_M_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_re_M_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_re_M_dot_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_M_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_M_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_re_M_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_re_M_dot_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_pM_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_pM_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_re_pM_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_re_pM_dot_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_pM_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_pM_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_re_pM_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_re_pM_dot_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_M_dot_Ma (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_M_dot_Ma(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_M_dot_pMa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_M_dot_pMa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_pM_dot_Ma (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_pM_dot_Ma(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_pM_dot_pMa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_pM_dot_pMa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_Ma_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_Ma_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_Ma_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_Ma_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_pMa_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_pMa_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_pMa_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_pMa_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_norm2_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_norm2_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_vpeq_norm2_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_norm2_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_C_vmeq_M_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_M_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_re_M_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_re_M_dot_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_M_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_M_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_re_M_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_re_M_dot_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_pM_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_pM_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_re_pM_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_re_pM_dot_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_pM_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_pM_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_re_pM_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_re_pM_dot_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_M_dot_Ma (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_M_dot_Ma(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_M_dot_pMa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_M_dot_pMa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_pM_dot_Ma (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_pM_dot_Ma(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_pM_dot_pMa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_pM_dot_pMa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_Ma_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_Ma_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_Ma_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_Ma_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_pMa_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_pMa_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_pMa_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_pMa_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_norm2_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_norm2_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_vmeq_norm2_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_norm2_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_C_veqm_M_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_M_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_re_M_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_re_M_dot_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_M_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_M_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_re_M_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_re_M_dot_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_pM_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_pM_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_re_pM_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_re_pM_dot_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_pM_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_pM_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_re_pM_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_re_pM_dot_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_M_dot_Ma (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_M_dot_Ma(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_M_dot_pMa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_M_dot_pMa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_pM_dot_Ma (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_pM_dot_Ma(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_pM_dot_pMa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_pM_dot_pMa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_Ma_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_Ma_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_Ma_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_Ma_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_pMa_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_pMa_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_pMa_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_pMa_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_norm2_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_norm2_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_veqm_norm2_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_norm2_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_C_xeq_M_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_M_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_re_M_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_re_M_dot_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_M_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_M_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_re_M_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_re_M_dot_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_pM_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_pM_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_re_pM_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_re_pM_dot_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_pM_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_pM_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_re_pM_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_re_pM_dot_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_M_dot_Ma (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_M_dot_Ma(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_M_dot_pMa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_M_dot_pMa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_pM_dot_Ma (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_pM_dot_Ma(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_pM_dot_pMa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_pM_dot_pMa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_Ma_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_Ma_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_Ma_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_Ma_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_pMa_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_pMa_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_pMa_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_pMa_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_norm2_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_norm2_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xeq_norm2_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_norm2_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_C_xpeq_M_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_M_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_re_M_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_re_M_dot_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_M_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_M_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_re_M_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_re_M_dot_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_pM_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_pM_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_re_pM_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_re_pM_dot_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_pM_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_pM_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_re_pM_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_re_pM_dot_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_M_dot_Ma (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_M_dot_Ma(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_M_dot_pMa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_M_dot_pMa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_pM_dot_Ma (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_pM_dot_Ma(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_pM_dot_pMa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_pM_dot_pMa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_Ma_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_Ma_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_Ma_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_Ma_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_pMa_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_pMa_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_pMa_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_pMa_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_norm2_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_norm2_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xpeq_norm2_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_norm2_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_C_xmeq_M_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_M_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_re_M_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_re_M_dot_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_M_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_M_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_re_M_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_re_M_dot_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_pM_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_pM_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_re_pM_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_re_pM_dot_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_pM_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_pM_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_re_pM_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_re_pM_dot_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_M_dot_Ma (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_M_dot_Ma(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_M_dot_pMa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_M_dot_pMa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_pM_dot_Ma (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_pM_dot_Ma(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_pM_dot_pMa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_pM_dot_pMa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_Ma_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_Ma_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_Ma_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_Ma_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_pMa_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_pMa_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_pMa_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_pMa_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_norm2_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_norm2_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xmeq_norm2_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_norm2_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_C_xeqm_M_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_M_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_re_M_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_re_M_dot_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_M_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_M_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_re_M_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_re_M_dot_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_pM_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_pM_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_re_pM_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_re_pM_dot_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_pM_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_pM_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_re_pM_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_re_pM_dot_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_M_dot_Ma (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_M_dot_Ma(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_M_dot_pMa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_M_dot_pMa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_pM_dot_Ma (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_pM_dot_Ma(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_pM_dot_pMa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_pM_dot_pMa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_Ma_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_Ma_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_Ma_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_Ma_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_pMa_dot_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_pMa_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_pMa_dot_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_pMa_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_norm2_M (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_norm2_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xeqm_norm2_pM (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_norm2_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_C_veq_P_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_P_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_re_P_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_re_P_dot_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_P_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_P_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_re_P_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_re_P_dot_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_pP_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_pP_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_re_pP_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_re_pP_dot_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_pP_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_pP_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_re_pP_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_re_pP_dot_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_P_dot_Pa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_P_dot_Pa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_P_dot_pPa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_P_dot_pPa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_pP_dot_Pa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_pP_dot_Pa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_pP_dot_pPa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_pP_dot_pPa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_Pa_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_Pa_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_Pa_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_Pa_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_pPa_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_pPa_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veq_pPa_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veq_pPa_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veq_norm2_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_norm2_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_veq_norm2_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veq_norm2_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_C_vpeq_P_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_P_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_re_P_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_re_P_dot_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_P_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_P_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_re_P_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_re_P_dot_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_pP_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_pP_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_re_pP_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_re_pP_dot_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_pP_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_pP_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_re_pP_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_re_pP_dot_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_P_dot_Pa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_P_dot_Pa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_P_dot_pPa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_P_dot_pPa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_pP_dot_Pa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_pP_dot_Pa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_pP_dot_pPa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_pP_dot_pPa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_Pa_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_Pa_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_Pa_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_Pa_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_pPa_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_pPa_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vpeq_pPa_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vpeq_pPa_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vpeq_norm2_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_norm2_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_vpeq_norm2_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vpeq_norm2_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_C_vmeq_P_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_P_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_re_P_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_re_P_dot_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_P_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_P_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_re_P_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_re_P_dot_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_pP_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_pP_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_re_pP_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_re_pP_dot_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_pP_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_pP_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_re_pP_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_re_pP_dot_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_P_dot_Pa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_P_dot_Pa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_P_dot_pPa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_P_dot_pPa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_pP_dot_Pa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_pP_dot_Pa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_pP_dot_pPa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_pP_dot_pPa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_Pa_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_Pa_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_Pa_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_Pa_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_pPa_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_pPa_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_vmeq_pPa_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_vmeq_pPa_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_vmeq_norm2_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_norm2_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_vmeq_norm2_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_vmeq_norm2_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_C_veqm_P_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_P_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_re_P_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_re_P_dot_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_P_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_P_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_re_P_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_re_P_dot_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_pP_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_pP_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_re_pP_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_re_pP_dot_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_pP_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_pP_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_re_pP_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_re_pP_dot_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_P_dot_Pa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_P_dot_Pa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_P_dot_pPa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_P_dot_pPa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_pP_dot_Pa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_pP_dot_Pa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_pP_dot_pPa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_pP_dot_pPa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_Pa_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_Pa_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_Pa_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_Pa_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_pPa_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_pPa_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_C_veqm_pPa_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_veqm_pPa_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_R_veqm_norm2_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_norm2_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_veqm_norm2_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_veqm_norm2_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_C_xeq_P_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_P_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_re_P_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_re_P_dot_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_P_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_P_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_re_P_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_re_P_dot_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_pP_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_pP_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_re_pP_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_re_pP_dot_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_pP_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_pP_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_re_pP_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_re_pP_dot_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_P_dot_Pa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_P_dot_Pa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_P_dot_pPa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_P_dot_pPa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_pP_dot_Pa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_pP_dot_Pa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_pP_dot_pPa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_pP_dot_pPa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_Pa_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_Pa_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_Pa_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_Pa_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_pPa_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_pPa_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeq_pPa_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeq_pPa_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeq_norm2_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_norm2_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xeq_norm2_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeq_norm2_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_C_xpeq_P_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_P_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_re_P_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_re_P_dot_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_P_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_P_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_re_P_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_re_P_dot_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_pP_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_pP_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_re_pP_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_re_pP_dot_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_pP_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_pP_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_re_pP_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_re_pP_dot_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_P_dot_Pa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_P_dot_Pa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_P_dot_pPa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_P_dot_pPa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_pP_dot_Pa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_pP_dot_Pa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_pP_dot_pPa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_pP_dot_pPa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_Pa_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_Pa_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_Pa_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_Pa_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_pPa_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_pPa_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xpeq_pPa_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xpeq_pPa_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xpeq_norm2_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_norm2_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xpeq_norm2_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xpeq_norm2_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_C_xmeq_P_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_P_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_re_P_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_re_P_dot_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_P_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_P_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_re_P_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_re_P_dot_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_pP_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_pP_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_re_pP_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_re_pP_dot_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_pP_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_pP_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_re_pP_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_re_pP_dot_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_P_dot_Pa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_P_dot_Pa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_P_dot_pPa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_P_dot_pPa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_pP_dot_Pa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_pP_dot_Pa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_pP_dot_pPa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_pP_dot_pPa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_Pa_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_Pa_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_Pa_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_Pa_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_pPa_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_pPa_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xmeq_pPa_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xmeq_pPa_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xmeq_norm2_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_norm2_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xmeq_norm2_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xmeq_norm2_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_C_xeqm_P_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_P_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_re_P_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_re_P_dot_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_P_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_P_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_re_P_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_re_P_dot_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_pP_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_pP_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_re_pP_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_re_pP_dot_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_pP_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_pP_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_re_pP_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_re_pP_dot_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_P_dot_Pa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_P_dot_Pa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_P_dot_pPa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_P_dot_pPa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_pP_dot_Pa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_pP_dot_Pa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_pP_dot_pPa (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_pP_dot_pPa(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_Pa_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_Pa_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_Pa_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_Pa_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_pPa_dot_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_pPa_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_C_xeqm_pPa_dot_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_C_xeqm_pPa_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_R_xeqm_norm2_P (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_norm2_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xeqm_norm2_pP (lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)) */
void QLA_FN_R_xeqm_norm2_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_M_veq_V_times_Va (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_veq_V_times_Va(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_V_times_pVa (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_veq_V_times_pVa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_pV_times_Va (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_veq_pV_times_Va(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_pV_times_pVa (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_veq_pV_times_pVa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_V_times_Va (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_vpeq_V_times_Va(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_V_times_pVa (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_vpeq_V_times_pVa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_pV_times_Va (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_vpeq_pV_times_Va(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vpeq_pV_times_pVa (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_vpeq_pV_times_pVa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_V_times_Va (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_vmeq_V_times_Va(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_V_times_pVa (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_vmeq_V_times_pVa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_pV_times_Va (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_vmeq_pV_times_Va(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_vmeq_pV_times_pVa (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_vmeq_pV_times_pVa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veqm_V_times_Va (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_veqm_V_times_Va(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veqm_V_times_pVa (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_veqm_V_times_pVa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veqm_pV_times_Va (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_veqm_pV_times_Va(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veqm_pV_times_pVa (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_veqm_pV_times_pVa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_xeq_V_times_Va (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_xeq_V_times_Va(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_V_times_pVa (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_xeq_V_times_pVa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pV_times_Va (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_xeq_pV_times_Va(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pV_times_pVa (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_xeq_pV_times_pVa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_V_times_Va (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_xpeq_V_times_Va(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_V_times_pVa (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_xpeq_V_times_pVa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_pV_times_Va (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_xpeq_pV_times_Va(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xpeq_pV_times_pVa (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_xpeq_pV_times_pVa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_V_times_Va (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_xmeq_V_times_Va(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_V_times_pVa (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_xmeq_V_times_pVa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_pV_times_Va (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_xmeq_pV_times_Va(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xmeq_pV_times_pVa (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_xmeq_pV_times_pVa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_V_times_Va (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_xeqm_V_times_Va(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_V_times_pVa (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_xeqm_V_times_pVa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_pV_times_Va (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_xeqm_pV_times_Va(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeqm_pV_times_pVa (lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)) */
void QLA_FN_M_xeqm_pV_times_pVa(int nc, void * r, void * a, void * b, int * index, int n);
/* ---- fill: replaces the FN functions emitted by lib/perl/build_qla.pl:2561-2618 (zero fills */
/* replaces QLA_FN_V_veq_v (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_V_veq_v(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_vpeq_v (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_V_vpeq_v(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_vmeq_v (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_V_vmeq_v(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_veqm_v (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_V_veqm_v(int nc, void * r, void * a, int n);
/* replaces QLA_FN_V_veq_zero (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_V_veq_zero(int nc, void * r, int n);
/* ---- random: replaces the FN functions emitted by lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills */
/* replaces QLA_FN_V_veq_gaussian_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_FN_V_veq_gaussian_S(int nc, void * r, QLA_RandomState *QLA_B200_RESTRICT a, int n);
/* replaces QLA_FN_V_veq_gaussian_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_FN_V_veq_gaussian_pS(int nc, void * r, QLA_RandomState *QLA_B200_RESTRICT * a, int n);
/* ---- mask: replaces the FN functions emitted by lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero) */
/* replaces QLA_FN_V_veq_V_mask_I (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_V_veq_V_mask_I(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_FN_V_veq_V_mask_pI (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_V_veq_V_mask_pI(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_FN_V_veq_pV_mask_I (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_V_veq_pV_mask_I(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_FN_V_veq_pV_mask_pI (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_V_veq_pV_mask_pI(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* ---- fill: replaces the FN functions emitted by lib/perl/build_qla.pl:2561-2618 (zero fills */
/* replaces QLA_FN_H_veq_h (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_H_veq_h(int nc, void * r, void * a, int n);
/* replaces QLA_FN_H_vpeq_h (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_H_vpeq_h(int nc, void * r, void * a, int n);
/* replaces QLA_FN_H_vmeq_h (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_H_vmeq_h(int nc, void * r, void * a, int n);
/* replaces QLA_FN_H_veqm_h (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_H_veqm_h(int nc, void * r, void * a, int n);
/* replaces QLA_FN_H_veq_zero (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_H_veq_zero(int nc, void * r, int n);
/* ---- random: replaces the FN functions emitted by lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills */
/* replaces QLA_FN_H_veq_gaussian_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_FN_H_veq_gaussian_S(int nc, void * r, QLA_RandomState *QLA_B200_RESTRICT a, int n);
/* replaces QLA_FN_H_veq_gaussian_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_FN_H_veq_gaussian_pS(int nc, void * r, QLA_RandomState *QLA_B200_RESTRICT * a, int n);
/* ---- mask: replaces the FN functions emitted by lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero) */
/* replaces QLA_FN_H_veq_H_mask_I (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_H_veq_H_mask_I(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_FN_H_veq_H_mask_pI (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_H_veq_H_mask_pI(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_FN_H_veq_pH_mask_I (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_H_veq_pH_mask_I(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_FN_H_veq_pH_mask_pI (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_H_veq_pH_mask_pI(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* ---- fill: replaces the FN functions emitted by lib/perl/build_qla.pl:2561-2618 (zero fills */
/* replaces QLA_FN_D_veq_d (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_D_veq_d(int nc, void * r, void * a, int n);
/* replaces QLA_FN_D_vpeq_d (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_D_vpeq_d(int nc, void * r, void * a, int n);
/* replaces QLA_FN_D_vmeq_d (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_D_vmeq_d(int nc, void * r, void * a, int n);
/* replaces QLA_FN_D_veqm_d (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_D_veqm_d(int nc, void * r, void * a, int n);
/* replaces QLA_FN_D_veq_zero (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_D_veq_zero(int nc, void * r, int n);
/* ---- random: replaces the FN functions emitted by lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills */
/* replaces QLA_FN_D_veq_gaussian_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_FN_D_veq_gaussian_S(int nc, void * r, QLA_RandomState *QLA_B200_RESTRICT a, int n);
/* replaces QLA_FN_D_veq_gaussian_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_FN_D_veq_gaussian_pS(int nc, void * r, QLA_RandomState *QLA_B200_RESTRICT * a, int n);
/* ---- mask: replaces the FN functions emitted by lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero) */
/* replaces QLA_FN_D_veq_D_mask_I (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_D_veq_D_mask_I(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_FN_D_veq_D_mask_pI (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_D_veq_D_mask_pI(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_FN_D_veq_pD_mask_I (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_D_veq_pD_mask_I(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_FN_D_veq_pD_mask_pI (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_D_veq_pD_mask_pI(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* ---- fill: replaces the FN functions emitted by lib/perl/build_qla.pl:2561-2618 (zero fills */
/* replaces QLA_FN_M_veq_m (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_M_veq_m(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_vpeq_m (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_M_vpeq_m(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_vmeq_m (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_M_vmeq_m(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veqm_m (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_M_veqm_m(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_zero (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_M_veq_zero(int nc, void * r, int n);
/* ---- random: replaces the FN functions emitted by lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills */
/* replaces QLA_FN_M_veq_gaussian_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_FN_M_veq_gaussian_S(int nc, void * r, QLA_RandomState *QLA_B200_RESTRICT a, int n);
/* replaces QLA_FN_M_veq_gaussian_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_FN_M_veq_gaussian_pS(int nc, void * r, QLA_RandomState *QLA_B200_RESTRICT * a, int n);
/* ---- mask: replaces the FN functions emitted by lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero) */
/* replaces QLA_FN_M_veq_M_mask_I (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_M_veq_M_mask_I(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_FN_M_veq_M_mask_pI (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_M_veq_M_mask_pI(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_FN_M_veq_pM_mask_I (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_M_veq_pM_mask_I(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_FN_M_veq_pM_mask_pI (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_M_veq_pM_mask_pI(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* ---- fill: replaces the FN functions emitted by lib/perl/build_qla.pl:2561-2618 (zero fills */
/* replaces QLA_FN_P_veq_p (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_P_veq_p(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_vpeq_p (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_P_vpeq_p(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_vmeq_p (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_P_vmeq_p(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_veqm_p (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_P_veqm_p(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_veq_zero (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_P_veq_zero(int nc, void * r, int n);
/* ---- random: replaces the FN functions emitted by lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills */
/* replaces QLA_FN_P_veq_gaussian_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_FN_P_veq_gaussian_S(int nc, void * r, QLA_RandomState *QLA_B200_RESTRICT a, int n);
/* replaces QLA_FN_P_veq_gaussian_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_FN_P_veq_gaussian_pS(int nc, void * r, QLA_RandomState *QLA_B200_RESTRICT * a, int n);
/* ---- mask: replaces the FN functions emitted by lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero) */
/* replaces QLA_FN_P_veq_P_mask_I (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_P_veq_P_mask_I(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_FN_P_veq_P_mask_pI (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_P_veq_P_mask_pI(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_FN_P_veq_pP_mask_I (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_P_veq_pP_mask_I(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT b, int n);
/* replaces QLA_FN_P_veq_pP_mask_pI (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_P_veq_pP_mask_pI(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT * b, int n);
/* ---- fill: replaces the FN functions emitted by lib/perl/build_qla.pl:2561-2618 (zero fills */
/* replaces QLA_FN_M_veq_c (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_M_veq_c(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_FN_M_vpeq_c (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_M_vpeq_c(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_FN_M_vmeq_c (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_M_vmeq_c(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* replaces QLA_FN_M_veqm_c (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_M_veqm_c(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, int n);
/* ---- component: replaces the FN functions emitted by lib/perl/build_qla.pl:767-931 (array components */
/* replaces QLA_FN_C_veq_elem_V (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_C_veq_elem_V(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int i_c, int n);
/* replaces QLA_FN_V_veq_elem_C (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_V_veq_elem_C(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, int i_c, int n);
/* replaces QLA_FN_C_veq_elem_pV (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_C_veq_elem_pV(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int i_c, int n);
/* replaces QLA_FN_V_veq_elem_pC (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_V_veq_elem_pC(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, int i_c, int n);
/* replaces QLA_FN_C_veq_elem_H (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_C_veq_elem_H(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int i_c, int i_s, int n);
/* replaces QLA_FN_H_veq_elem_C (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_H_veq_elem_C(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, int i_c, int i_s, int n);
/* replaces QLA_FN_C_veq_elem_pH (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_C_veq_elem_pH(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int i_c, int i_s, int n);
/* replaces QLA_FN_H_veq_elem_pC (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_H_veq_elem_pC(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, int i_c, int i_s, int n);
/* replaces QLA_FN_C_veq_elem_D (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_C_veq_elem_D(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int i_c, int i_s, int n);
/* replaces QLA_FN_D_veq_elem_C (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_D_veq_elem_C(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, int i_c, int i_s, int n);
/* replaces QLA_FN_C_veq_elem_pD (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_C_veq_elem_pD(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int i_c, int i_s, int n);
/* replaces QLA_FN_D_veq_elem_pC (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_D_veq_elem_pC(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, int i_c, int i_s, int n);
/* replaces QLA_FN_C_veq_elem_M (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_C_veq_elem_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int i_c, int j_c, int n);
/* replaces QLA_FN_M_veq_elem_C (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_M_veq_elem_C(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, int i_c, int j_c, int n);
/* replaces QLA_FN_C_veq_elem_pM (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_C_veq_elem_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int i_c, int j_c, int n);
/* replaces QLA_FN_M_veq_elem_pC (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_M_veq_elem_pC(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, int i_c, int j_c, int n);
/* replaces QLA_FN_C_veq_elem_P (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_C_veq_elem_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int i_c, int i_s, int j_c, int j_s, int n);
/* replaces QLA_FN_P_veq_elem_C (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_P_veq_elem_C(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, int i_c, int i_s, int j_c, int j_s, int n);
/* replaces QLA_FN_C_veq_elem_pP (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_C_veq_elem_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int i_c, int i_s, int j_c, int j_s, int n);
/* replaces QLA_FN_P_veq_elem_pC (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_P_veq_elem_pC(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, int i_c, int i_s, int j_c, int j_s, int n);
/* replaces QLA_FN_V_veq_colorvec_H (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_V_veq_colorvec_H(int nc, void * r, void * a, int i_s, int n);
/* replaces QLA_FN_H_veq_colorvec_V (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_H_veq_colorvec_V(int nc, void * r, void * a, int i_s, int n);
/* replaces QLA_FN_V_veq_colorvec_pH (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_V_veq_colorvec_pH(int nc, void * r, void * a, int i_s, int n);
/* replaces QLA_FN_H_veq_colorvec_pV (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_H_veq_colorvec_pV(int nc, void * r, void * a, int i_s, int n);
/* replaces QLA_FN_V_veq_colorvec_D (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_V_veq_colorvec_D(int nc, void * r, void * a, int i_s, int n);
/* replaces QLA_FN_D_veq_colorvec_V (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_D_veq_colorvec_V(int nc, void * r, void * a, int i_s, int n);
/* replaces QLA_FN_V_veq_colorvec_pD (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_V_veq_colorvec_pD(int nc, void * r, void * a, int i_s, int n);
/* replaces QLA_FN_D_veq_colorvec_pV (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_D_veq_colorvec_pV(int nc, void * r, void * a, int i_s, int n);
/* replaces QLA_FN_V_veq_colorvec_M (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_V_veq_colorvec_M(int nc, void * r, void * a, int j_c, int n);
/* replaces QLA_FN_M_veq_colorvec_V (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_M_veq_colorvec_V(int nc, void * r, void * a, int j_c, int n);
/* replaces QLA_FN_V_veq_colorvec_pM (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_V_veq_colorvec_pM(int nc, void * r, void * a, int j_c, int n);
/* replaces QLA_FN_M_veq_colorvec_pV (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_M_veq_colorvec_pV(int nc, void * r, void * a, int j_c, int n);
/* replaces QLA_FN_V_veq_colorvec_P (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_V_veq_colorvec_P(int nc, void * r, void * a, int i_s, int j_c, int j_s, int n);
/* replaces QLA_FN_P_veq_colorvec_V (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_P_veq_colorvec_V(int nc, void * r, void * a, int i_s, int j_c, int j_s, int n);
/* replaces QLA_FN_V_veq_colorvec_pP (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_V_veq_colorvec_pP(int nc, void * r, void * a, int i_s, int j_c, int j_s, int n);
/* replaces QLA_FN_P_veq_colorvec_pV (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_P_veq_colorvec_pV(int nc, void * r, void * a, int i_s, int j_c, int j_s, int n);
/* replaces QLA_FN_D_veq_diracvec_P (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_D_veq_diracvec_P(int nc, void * r, void * a, int j_c, int j_s, int n);
/* replaces QLA_FN_P_veq_diracvec_D (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_P_veq_diracvec_D(int nc, void * r, void * a, int j_c, int j_s, int n);
/* replaces QLA_FN_D_veq_diracvec_pP (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_D_veq_diracvec_pP(int nc, void * r, void * a, int j_c, int j_s, int n);
/* replaces QLA_FN_P_veq_diracvec_pD (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_P_veq_diracvec_pD(int nc, void * r, void * a, int j_c, int j_s, int n);
/* ---- gamma: replaces the FN functions emitted by lib/perl/build_qla.pl:1358-1412 (left / right multiplication by gamma_mu */
/* replaces QLA_FN_D_veq_gamma_times_D (lib/perl/build_qla.pl:1358-1412 (left / right multiplication by gamma_mu, mu = 0..15), expressions_gamma.pl:59-134, 384-470) */
void QLA_FN_D_veq_gamma_times_D(int nc, void * r, void * a, int mu, int n);
/* replaces QLA_FN_D_veq_gamma_times_pD (lib/perl/build_qla.pl:1358-1412 (left / right multiplication by gamma_mu, mu = 0..15), expressions_gamma.pl:59-134, 384-470) */
void QLA_FN_D_veq_gamma_times_pD(int nc, void * r, void * a, int mu, int n);
/* replaces QLA_FN_P_veq_gamma_times_P (lib/perl/build_qla.pl:1358-1412 (left / right multiplication by gamma_mu, mu = 0..15), expressions_gamma.pl:59-134, 384-470) */
void QLA_FN_P_veq_gamma_times_P(int nc, void * r, void * a, int mu, int n);
/* replaces QLA_FN_P_veq_gamma_times_pP (lib/perl/build_qla.pl:1358-1412 (left / right multiplication by gamma_mu, mu = 0..15), expressions_gamma.pl:59-134, 384-470) */
void QLA_FN_P_veq_gamma_times_pP(int nc, void * r, void * a, int mu, int n);
/* replaces QLA_FN_P_veq_P_times_gamma (lib/perl/build_qla.pl:1358-1412 (left / right multiplication by gamma_mu, mu = 0..15), expressions_gamma.pl:59-134, 384-470) */
void QLA_FN_P_veq_P_times_gamma(int nc, void * r, void * a, int mu, int n);
/* replaces QLA_FN_P_veq_pP_times_gamma (lib/perl/build_qla.pl:1358-1412 (left / right multiplication by gamma_mu, mu = 0..15), expressions_gamma.pl:59-134, 384-470) */
void QLA_FN_P_veq_pP_times_gamma(int nc, void * r, void * a, int mu, int n);
/* ---- trace: replaces the FN functions emitted by lib/perl/build_qla.pl:933-1064 (trace */
/* replaces QLA_FN_C_veq_trace_M (lib/perl/build_qla.pl:933-1064 (trace, real / imaginary trace, traceless antihermitian part)) */
void QLA_FN_C_veq_trace_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_veq_re_trace_M (lib/perl/build_qla.pl:933-1064 (trace, real / imaginary trace, traceless antihermitian part)) */
void QLA_FN_R_veq_re_trace_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_veq_im_trace_M (lib/perl/build_qla.pl:933-1064 (trace, real / imaginary trace, traceless antihermitian part)) */
void QLA_FN_R_veq_im_trace_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_M_veq_antiherm_M (lib/perl/build_qla.pl:933-1064 (trace, real / imaginary trace, traceless antihermitian part)) */
void QLA_FN_M_veq_antiherm_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_C_veq_trace_pM (lib/perl/build_qla.pl:933-1064 (trace, real / imaginary trace, traceless antihermitian part)) */
void QLA_FN_C_veq_trace_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_veq_re_trace_pM (lib/perl/build_qla.pl:933-1064 (trace, real / imaginary trace, traceless antihermitian part)) */
void QLA_FN_R_veq_re_trace_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_R_veq_im_trace_pM (lib/perl/build_qla.pl:933-1064 (trace, real / imaginary trace, traceless antihermitian part)) */
void QLA_FN_R_veq_im_trace_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_M_veq_antiherm_pM (lib/perl/build_qla.pl:933-1064 (trace, real / imaginary trace, traceless antihermitian part)) */
void QLA_FN_M_veq_antiherm_pM(int nc, void * r, void * a, int n);
/* ---- gred: replaces the FN functions emitted by lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators */
/* replaces QLA_FN_c_veq_Ma_dot_M (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_veq_Ma_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_c_veq_Ma_dot_pM (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_veq_Ma_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_c_veq_pMa_dot_M (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_veq_pMa_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_c_veq_pMa_dot_pM (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_veq_pMa_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_c_veq_P_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_veq_P_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_c_veq_P_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_veq_P_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_c_veq_pP_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_veq_pP_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_c_veq_pP_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_veq_pP_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_c_veq_Pa_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_veq_Pa_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_c_veq_Pa_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_veq_Pa_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_c_veq_pPa_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_veq_pPa_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_c_veq_pPa_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_veq_pPa_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_r_veq_re_P_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_r_veq_re_P_dot_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_r_veq_re_P_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_r_veq_re_P_dot_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_r_veq_re_pP_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_r_veq_re_pP_dot_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_r_veq_re_pP_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_r_veq_re_pP_dot_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int n);
/* replaces QLA_FN_r_veq_norm2_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_r_veq_norm2_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* replaces QLA_FN_r_veq_norm2_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_r_veq_norm2_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int n);
/* ---- gsum: replaces the FN functions emitted by lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites) */
/* replaces QLA_FN_v_veq_sum_V (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_FN_v_veq_sum_V(int nc, void * r, void * a, int n);
/* replaces QLA_FN_v_veq_sum_pV (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_FN_v_veq_sum_pV(int nc, void * r, void * a, int n);
/* replaces QLA_FN_h_veq_sum_H (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_FN_h_veq_sum_H(int nc, void * r, void * a, int n);
/* replaces QLA_FN_h_veq_sum_pH (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_FN_h_veq_sum_pH(int nc, void * r, void * a, int n);
/* replaces QLA_FN_d_veq_sum_D (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_FN_d_veq_sum_D(int nc, void * r, void * a, int n);
/* replaces QLA_FN_d_veq_sum_pD (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_FN_d_veq_sum_pD(int nc, void * r, void * a, int n);
/* replaces QLA_FN_m_veq_sum_M (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_FN_m_veq_sum_M(int nc, void * r, void * a, int n);
/* replaces QLA_FN_m_veq_sum_pM (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_FN_m_veq_sum_pM(int nc, void * r, void * a, int n);
/* replaces QLA_FN_p_veq_sum_P (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_FN_p_veq_sum_P(int nc, void * r, void * a, int n);
/* replaces QLA_FN_p_veq_sum_pP (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_FN_p_veq_sum_pP(int nc, void * r, void * a, int n);
/* ---- fill: replaces the FN functions emitted by lib/perl/build_qla.pl:2561-2618 (zero fills */
/* replaces QLA_FN_V_xeq_v (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_V_xeq_v(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xpeq_v (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_V_xpeq_v(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xmeq_v (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_V_xmeq_v(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xeqm_v (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_V_xeqm_v(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_V_xeq_zero (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_V_xeq_zero(int nc, void * r, int * index, int n);
/* ---- random: replaces the FN functions emitted by lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills */
/* replaces QLA_FN_V_xeq_gaussian_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_FN_V_xeq_gaussian_S(int nc, void * r, QLA_RandomState *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_FN_V_xeq_gaussian_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_FN_V_xeq_gaussian_pS(int nc, void * r, QLA_RandomState *QLA_B200_RESTRICT * a, int * index, int n);
/* ---- mask: replaces the FN functions emitted by lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero) */
/* replaces QLA_FN_V_xeq_V_mask_I (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_V_xeq_V_mask_I(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_FN_V_xeq_V_mask_pI (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_V_xeq_V_mask_pI(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_FN_V_xeq_pV_mask_I (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_V_xeq_pV_mask_I(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_FN_V_xeq_pV_mask_pI (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_V_xeq_pV_mask_pI(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* ---- fill: replaces the FN functions emitted by lib/perl/build_qla.pl:2561-2618 (zero fills */
/* replaces QLA_FN_H_xeq_h (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_H_xeq_h(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_H_xpeq_h (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_H_xpeq_h(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_H_xmeq_h (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_H_xmeq_h(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_H_xeqm_h (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_H_xeqm_h(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_H_xeq_zero (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_H_xeq_zero(int nc, void * r, int * index, int n);
/* ---- random: replaces the FN functions emitted by lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills */
/* replaces QLA_FN_H_xeq_gaussian_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_FN_H_xeq_gaussian_S(int nc, void * r, QLA_RandomState *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_FN_H_xeq_gaussian_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_FN_H_xeq_gaussian_pS(int nc, void * r, QLA_RandomState *QLA_B200_RESTRICT * a, int * index, int n);
/* ---- mask: replaces the FN functions emitted by lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero) */
/* replaces QLA_FN_H_xeq_H_mask_I (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_H_xeq_H_mask_I(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_FN_H_xeq_H_mask_pI (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_H_xeq_H_mask_pI(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_FN_H_xeq_pH_mask_I (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_H_xeq_pH_mask_I(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_FN_H_xeq_pH_mask_pI (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_H_xeq_pH_mask_pI(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* ---- fill: replaces the FN functions emitted by lib/perl/build_qla.pl:2561-2618 (zero fills */
/* replaces QLA_FN_D_xeq_d (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_D_xeq_d(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_D_xpeq_d (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_D_xpeq_d(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_D_xmeq_d (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_D_xmeq_d(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_D_xeqm_d (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_D_xeqm_d(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_D_xeq_zero (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_D_xeq_zero(int nc, void * r, int * index, int n);
/* ---- random: replaces the FN functions emitted by lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills */
/* replaces QLA_FN_D_xeq_gaussian_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_FN_D_xeq_gaussian_S(int nc, void * r, QLA_RandomState *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_FN_D_xeq_gaussian_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_FN_D_xeq_gaussian_pS(int nc, void * r, QLA_RandomState *QLA_B200_RESTRICT * a, int * index, int n);
/* ---- mask: replaces the FN functions emitted by lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero) */
/* replaces QLA_FN_D_xeq_D_mask_I (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_D_xeq_D_mask_I(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_FN_D_xeq_D_mask_pI (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_D_xeq_D_mask_pI(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_FN_D_xeq_pD_mask_I (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_D_xeq_pD_mask_I(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_FN_D_xeq_pD_mask_pI (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_D_xeq_pD_mask_pI(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* ---- fill: replaces the FN functions emitted by lib/perl/build_qla.pl:2561-2618 (zero fills */
/* replaces QLA_FN_M_xeq_m (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_M_xeq_m(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xpeq_m (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_M_xpeq_m(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xmeq_m (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_M_xmeq_m(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeqm_m (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_M_xeqm_m(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_zero (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_M_xeq_zero(int nc, void * r, int * index, int n);
/* ---- random: replaces the FN functions emitted by lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills */
/* replaces QLA_FN_M_xeq_gaussian_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_FN_M_xeq_gaussian_S(int nc, void * r, QLA_RandomState *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_FN_M_xeq_gaussian_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_FN_M_xeq_gaussian_pS(int nc, void * r, QLA_RandomState *QLA_B200_RESTRICT * a, int * index, int n);
/* ---- mask: replaces the FN functions emitted by lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero) */
/* replaces QLA_FN_M_xeq_M_mask_I (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_M_xeq_M_mask_I(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_FN_M_xeq_M_mask_pI (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_M_xeq_M_mask_pI(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_FN_M_xeq_pM_mask_I (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_M_xeq_pM_mask_I(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_FN_M_xeq_pM_mask_pI (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_M_xeq_pM_mask_pI(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* ---- fill: replaces the FN functions emitted by lib/perl/build_qla.pl:2561-2618 (zero fills */
/* replaces QLA_FN_P_xeq_p (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_P_xeq_p(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xpeq_p (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_P_xpeq_p(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xmeq_p (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_P_xmeq_p(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xeqm_p (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_P_xeqm_p(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xeq_zero (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_P_xeq_zero(int nc, void * r, int * index, int n);
/* ---- random: replaces the FN functions emitted by lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills */
/* replaces QLA_FN_P_xeq_gaussian_S (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_FN_P_xeq_gaussian_S(int nc, void * r, QLA_RandomState *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_FN_P_xeq_gaussian_pS (lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36) */
void QLA_FN_P_xeq_gaussian_pS(int nc, void * r, QLA_RandomState *QLA_B200_RESTRICT * a, int * index, int n);
/* ---- mask: replaces the FN functions emitted by lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero) */
/* replaces QLA_FN_P_xeq_P_mask_I (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_P_xeq_P_mask_I(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_FN_P_xeq_P_mask_pI (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_P_xeq_P_mask_pI(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pP_mask_I (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_P_xeq_pP_mask_I(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_FN_P_xeq_pP_mask_pI (lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)) */
void QLA_FN_P_xeq_pP_mask_pI(int nc, void * r, void * a, QLA_Int *QLA_B200_RESTRICT * b, int * index, int n);
/* ---- fill: replaces the FN functions emitted by lib/perl/build_qla.pl:2561-2618 (zero fills */
/* replaces QLA_FN_M_xeq_c (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_M_xeq_c(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_FN_M_xpeq_c (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_M_xpeq_c(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_FN_M_xmeq_c (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_M_xmeq_c(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_FN_M_xeqm_c (lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), make_code_unary.pl (identity, diagfill, zero)) */
void QLA_FN_M_xeqm_c(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, int * index, int n);
/* ---- component: replaces the FN functions emitted by lib/perl/build_qla.pl:767-931 (array components */
/* replaces QLA_FN_C_xeq_elem_V (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_C_xeq_elem_V(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int i_c, int * index, int n);
/* replaces QLA_FN_V_xeq_elem_C (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_V_xeq_elem_C(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, int i_c, int * index, int n);
/* replaces QLA_FN_C_xeq_elem_pV (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_C_xeq_elem_pV(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int i_c, int * index, int n);
/* replaces QLA_FN_V_xeq_elem_pC (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_V_xeq_elem_pC(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, int i_c, int * index, int n);
/* replaces QLA_FN_C_xeq_elem_H (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_C_xeq_elem_H(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int i_c, int i_s, int * index, int n);
/* replaces QLA_FN_H_xeq_elem_C (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_H_xeq_elem_C(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, int i_c, int i_s, int * index, int n);
/* replaces QLA_FN_C_xeq_elem_pH (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_C_xeq_elem_pH(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int i_c, int i_s, int * index, int n);
/* replaces QLA_FN_H_xeq_elem_pC (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_H_xeq_elem_pC(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, int i_c, int i_s, int * index, int n);
/* replaces QLA_FN_C_xeq_elem_D (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_C_xeq_elem_D(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int i_c, int i_s, int * index, int n);
/* replaces QLA_FN_D_xeq_elem_C (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_D_xeq_elem_C(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, int i_c, int i_s, int * index, int n);
/* replaces QLA_FN_C_xeq_elem_pD (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_C_xeq_elem_pD(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int i_c, int i_s, int * index, int n);
/* replaces QLA_FN_D_xeq_elem_pC (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_D_xeq_elem_pC(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, int i_c, int i_s, int * index, int n);
/* replaces QLA_FN_C_xeq_elem_M (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_C_xeq_elem_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int i_c, int j_c, int * index, int n);
/* replaces QLA_FN_M_xeq_elem_C (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_M_xeq_elem_C(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, int i_c, int j_c, int * index, int n);
/* replaces QLA_FN_C_xeq_elem_pM (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_C_xeq_elem_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int i_c, int j_c, int * index, int n);
/* replaces QLA_FN_M_xeq_elem_pC (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_M_xeq_elem_pC(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, int i_c, int j_c, int * index, int n);
/* replaces QLA_FN_C_xeq_elem_P (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_C_xeq_elem_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int i_c, int i_s, int j_c, int j_s, int * index, int n);
/* replaces QLA_FN_P_xeq_elem_C (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_P_xeq_elem_C(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT a, int i_c, int i_s, int j_c, int j_s, int * index, int n);
/* replaces QLA_FN_C_xeq_elem_pP (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_C_xeq_elem_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int i_c, int i_s, int j_c, int j_s, int * index, int n);
/* replaces QLA_FN_P_xeq_elem_pC (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_P_xeq_elem_pC(int nc, void * r, QLA_F_Complex *QLA_B200_RESTRICT * a, int i_c, int i_s, int j_c, int j_s, int * index, int n);
/* replaces QLA_FN_V_xeq_colorvec_H (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_V_xeq_colorvec_H(int nc, void * r, void * a, int i_s, int * index, int n);
/* replaces QLA_FN_H_xeq_colorvec_V (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_H_xeq_colorvec_V(int nc, void * r, void * a, int i_s, int * index, int n);
/* replaces QLA_FN_V_xeq_colorvec_pH (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_V_xeq_colorvec_pH(int nc, void * r, void * a, int i_s, int * index, int n);
/* replaces QLA_FN_H_xeq_colorvec_pV (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_H_xeq_colorvec_pV(int nc, void * r, void * a, int i_s, int * index, int n);
/* replaces QLA_FN_V_xeq_colorvec_D (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_V_xeq_colorvec_D(int nc, void * r, void * a, int i_s, int * index, int n);
/* replaces QLA_FN_D_xeq_colorvec_V (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_D_xeq_colorvec_V(int nc, void * r, void * a, int i_s, int * index, int n);
/* replaces QLA_FN_V_xeq_colorvec_pD (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_V_xeq_colorvec_pD(int nc, void * r, void * a, int i_s, int * index, int n);
/* replaces QLA_FN_D_xeq_colorvec_pV (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_D_xeq_colorvec_pV(int nc, void * r, void * a, int i_s, int * index, int n);
/* replaces QLA_FN_V_xeq_colorvec_M (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_V_xeq_colorvec_M(int nc, void * r, void * a, int j_c, int * index, int n);
/* replaces QLA_FN_M_xeq_colorvec_V (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_M_xeq_colorvec_V(int nc, void * r, void * a, int j_c, int * index, int n);
/* replaces QLA_FN_V_xeq_colorvec_pM (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_V_xeq_colorvec_pM(int nc, void * r, void * a, int j_c, int * index, int n);
/* replaces QLA_FN_M_xeq_colorvec_pV (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_M_xeq_colorvec_pV(int nc, void * r, void * a, int j_c, int * index, int n);
/* replaces QLA_FN_V_xeq_colorvec_P (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_V_xeq_colorvec_P(int nc, void * r, void * a, int i_s, int j_c, int j_s, int * index, int n);
/* replaces QLA_FN_P_xeq_colorvec_V (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_P_xeq_colorvec_V(int nc, void * r, void * a, int i_s, int j_c, int j_s, int * index, int n);
/* replaces QLA_FN_V_xeq_colorvec_pP (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_V_xeq_colorvec_pP(int nc, void * r, void * a, int i_s, int j_c, int j_s, int * index, int n);
/* replaces QLA_FN_P_xeq_colorvec_pV (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_P_xeq_colorvec_pV(int nc, void * r, void * a, int i_s, int j_c, int j_s, int * index, int n);
/* replaces QLA_FN_D_xeq_diracvec_P (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_D_xeq_diracvec_P(int nc, void * r, void * a, int j_c, int j_s, int * index, int n);
/* replaces QLA_FN_P_xeq_diracvec_D (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_P_xeq_diracvec_D(int nc, void * r, void * a, int j_c, int j_s, int * index, int n);
/* replaces QLA_FN_D_xeq_diracvec_pP (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_D_xeq_diracvec_pP(int nc, void * r, void * a, int j_c, int j_s, int * index, int n);
/* replaces QLA_FN_P_xeq_diracvec_pD (lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: extraction and insertion)) */
void QLA_FN_P_xeq_diracvec_pD(int nc, void * r, void * a, int j_c, int j_s, int * index, int n);
/* ---- gamma: replaces the FN functions emitted by lib/perl/build_qla.pl:1358-1412 (left / right multiplication by gamma_mu */
/* replaces QLA_FN_D_xeq_gamma_times_D (lib/perl/build_qla.pl:1358-1412 (left / right multiplication by gamma_mu, mu = 0..15), expressions_gamma.pl:59-134, 384-470) */
void QLA_FN_D_xeq_gamma_times_D(int nc, void * r, void * a, int mu, int * index, int n);
/* replaces QLA_FN_D_xeq_gamma_times_pD (lib/perl/build_qla.pl:1358-1412 (left / right multiplication by gamma_mu, mu = 0..15), expressions_gamma.pl:59-134, 384-470) */
void QLA_FN_D_xeq_gamma_times_pD(int nc, void * r, void * a, int mu, int * index, int n);
/* replaces QLA_FN_P_xeq_gamma_times_P (lib/perl/build_qla.pl:1358-1412 (left / right multiplication by gamma_mu, mu = 0..15), expressions_gamma.pl:59-134, 384-470) */
void QLA_FN_P_xeq_gamma_times_P(int nc, void * r, void * a, int mu, int * index, int n);
/* replaces QLA_FN_P_xeq_gamma_times_pP (lib/perl/build_qla.pl:1358-1412 (left / right multiplication by gamma_mu, mu = 0..15), expressions_gamma.pl:59-134, 384-470) */
void QLA_FN_P_xeq_gamma_times_pP(int nc, void * r, void * a, int mu, int * index, int n);
/* replaces QLA_FN_P_xeq_P_times_gamma (lib/perl/build_qla.pl:1358-1412 (left / right multiplication by gamma_mu, mu = 0..15), expressions_gamma.pl:59-134, 384-470) */
void QLA_FN_P_xeq_P_times_gamma(int nc, void * r, void * a, int mu, int * index, int n);
/* replaces QLA_FN_P_xeq_pP_times_gamma (lib/perl/build_qla.pl:1358-1412 (left / right multiplication by gamma_mu, mu = 0..15), expressions_gamma.pl:59-134, 384-470) */
void QLA_FN_P_xeq_pP_times_gamma(int nc, void * r, void * a, int mu, int * index, int n);
/* ---- trace: replaces the FN functions emitted by lib/perl/build_qla.pl:933-1064 (trace */
/* replaces QLA_FN_C_xeq_trace_M (lib/perl/build_qla.pl:933-1064 (trace, real / imaginary trace, traceless antihermitian part)) */
void QLA_FN_C_xeq_trace_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xeq_re_trace_M (lib/perl/build_qla.pl:933-1064 (trace, real / imaginary trace, traceless antihermitian part)) */
void QLA_FN_R_xeq_re_trace_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xeq_im_trace_M (lib/perl/build_qla.pl:933-1064 (trace, real / imaginary trace, traceless antihermitian part)) */
void QLA_FN_R_xeq_im_trace_M(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_antiherm_M (lib/perl/build_qla.pl:933-1064 (trace, real / imaginary trace, traceless antihermitian part)) */
void QLA_FN_M_xeq_antiherm_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_C_xeq_trace_pM (lib/perl/build_qla.pl:933-1064 (trace, real / imaginary trace, traceless antihermitian part)) */
void QLA_FN_C_xeq_trace_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xeq_re_trace_pM (lib/perl/build_qla.pl:933-1064 (trace, real / imaginary trace, traceless antihermitian part)) */
void QLA_FN_R_xeq_re_trace_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_R_xeq_im_trace_pM (lib/perl/build_qla.pl:933-1064 (trace, real / imaginary trace, traceless antihermitian part)) */
void QLA_FN_R_xeq_im_trace_pM(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_antiherm_pM (lib/perl/build_qla.pl:933-1064 (trace, real / imaginary trace, traceless antihermitian part)) */
void QLA_FN_M_xeq_antiherm_pM(int nc, void * r, void * a, int * index, int n);
/* ---- gred: replaces the FN functions emitted by lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators */
/* replaces QLA_FN_c_xeq_Ma_dot_M (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_xeq_Ma_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_c_xeq_Ma_dot_pM (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_xeq_Ma_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_c_xeq_pMa_dot_M (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_xeq_pMa_dot_M(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_c_xeq_pMa_dot_pM (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_xeq_pMa_dot_pM(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_c_xeq_P_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_xeq_P_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_c_xeq_P_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_xeq_P_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_c_xeq_pP_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_xeq_pP_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_c_xeq_pP_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_xeq_pP_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_c_xeq_Pa_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_xeq_Pa_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_c_xeq_Pa_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_xeq_Pa_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_c_xeq_pPa_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_xeq_pPa_dot_P(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_c_xeq_pPa_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_c_xeq_pPa_dot_pP(int nc, QLA_F_Complex *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_r_xeq_re_P_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_r_xeq_re_P_dot_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_r_xeq_re_P_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_r_xeq_re_P_dot_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_r_xeq_re_pP_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_r_xeq_re_pP_dot_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_r_xeq_re_pP_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_r_xeq_re_pP_dot_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_r_xeq_norm2_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_r_xeq_norm2_P(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* replaces QLA_FN_r_xeq_norm2_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_FN_r_xeq_norm2_pP(int nc, QLA_F_Real *QLA_B200_RESTRICT r, void * a, int * index, int n);
/* ---- gsum: replaces the FN functions emitted by lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites) */
/* replaces QLA_FN_v_xeq_sum_V (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_FN_v_xeq_sum_V(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_v_xeq_sum_pV (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_FN_v_xeq_sum_pV(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_h_xeq_sum_H (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_FN_h_xeq_sum_H(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_h_xeq_sum_pH (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_FN_h_xeq_sum_pH(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_d_xeq_sum_D (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_FN_d_xeq_sum_D(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_d_xeq_sum_pD (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_FN_d_xeq_sum_pD(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_m_xeq_sum_M (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_FN_m_xeq_sum_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_m_xeq_sum_pM (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_FN_m_xeq_sum_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_p_xeq_sum_P (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_FN_p_xeq_sum_P(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_p_xeq_sum_pP (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_FN_p_xeq_sum_pP(int nc, void * r, void * a, int * index, int n);
/* ---- prop: replaces the FN functions emitted by lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products) */
/* replaces QLA_FN_P_veq_M_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_M_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_M_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_M_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_M_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_M_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_M_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_M_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_Ma_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_Ma_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_Ma_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_Ma_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_Ma_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_Ma_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_Ma_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_Ma_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pM_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pM_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pM_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pM_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pM_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pM_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pM_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pM_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pMa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pMa_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pMa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pMa_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pMa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pMa_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pMa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pMa_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_P_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_P_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_P_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_P_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_P_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_P_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_P_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_P_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_P_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_P_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_P_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_P_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_P_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_P_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_P_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_P_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_Pa_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_Pa_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_Pa_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_Pa_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_Pa_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_Pa_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_Pa_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_Pa_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_Pa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_Pa_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_Pa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_Pa_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_Pa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_Pa_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_Pa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_Pa_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pP_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pP_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pP_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pP_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pP_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pP_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pP_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pP_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pP_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pP_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pP_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pP_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pP_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pP_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pP_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pP_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pPa_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pPa_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pPa_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pPa_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pPa_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pPa_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pPa_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pPa_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pPa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pPa_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pPa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pPa_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pPa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pPa_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veq_pPa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veq_pPa_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_M_veq_spintrace_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_M_veq_spintrace_P(int nc, void * r, void * a, int n);
/* replaces QLA_FN_M_veq_spintrace_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_M_veq_spintrace_pP(int nc, void * r, void * a, int n);
/* replaces QLA_FN_P_vpeq_M_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_M_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_M_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_M_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_M_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_M_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_M_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_M_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_Ma_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_Ma_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_Ma_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_Ma_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_Ma_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_Ma_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_Ma_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_Ma_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pM_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pM_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pM_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pM_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pM_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pM_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pM_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pM_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pMa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pMa_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pMa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pMa_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pMa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pMa_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pMa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pMa_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_P_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_P_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_P_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_P_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_P_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_P_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_P_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_P_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_P_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_P_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_P_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_P_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_P_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_P_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_P_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_P_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_Pa_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_Pa_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_Pa_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_Pa_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_Pa_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_Pa_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_Pa_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_Pa_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_Pa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_Pa_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_Pa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_Pa_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_Pa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_Pa_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_Pa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_Pa_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pP_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pP_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pP_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pP_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pP_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pP_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pP_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pP_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pP_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pP_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pP_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pP_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pP_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pP_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pP_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pP_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pPa_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pPa_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pPa_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pPa_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pPa_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pPa_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pPa_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pPa_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pPa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pPa_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pPa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pPa_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pPa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pPa_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vpeq_pPa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vpeq_pPa_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_M_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_M_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_M_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_M_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_M_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_M_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_M_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_M_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_Ma_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_Ma_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_Ma_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_Ma_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_Ma_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_Ma_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_Ma_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_Ma_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pM_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pM_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pM_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pM_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pM_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pM_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pM_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pM_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pMa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pMa_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pMa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pMa_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pMa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pMa_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pMa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pMa_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_P_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_P_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_P_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_P_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_P_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_P_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_P_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_P_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_P_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_P_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_P_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_P_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_P_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_P_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_P_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_P_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_Pa_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_Pa_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_Pa_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_Pa_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_Pa_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_Pa_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_Pa_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_Pa_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_Pa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_Pa_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_Pa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_Pa_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_Pa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_Pa_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_Pa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_Pa_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pP_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pP_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pP_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pP_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pP_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pP_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pP_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pP_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pP_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pP_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pP_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pP_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pP_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pP_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pP_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pP_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pPa_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pPa_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pPa_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pPa_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pPa_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pPa_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pPa_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pPa_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pPa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pPa_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pPa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pPa_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pPa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pPa_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_vmeq_pPa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_vmeq_pPa_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_M_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_M_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_M_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_M_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_M_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_M_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_M_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_M_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_Ma_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_Ma_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_Ma_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_Ma_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_Ma_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_Ma_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_Ma_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_Ma_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pM_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pM_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pM_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pM_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pM_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pM_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pM_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pM_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pMa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pMa_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pMa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pMa_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pMa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pMa_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pMa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pMa_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_P_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_P_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_P_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_P_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_P_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_P_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_P_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_P_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_P_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_P_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_P_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_P_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_P_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_P_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_P_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_P_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_Pa_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_Pa_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_Pa_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_Pa_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_Pa_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_Pa_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_Pa_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_Pa_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_Pa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_Pa_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_Pa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_Pa_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_Pa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_Pa_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_Pa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_Pa_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pP_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pP_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pP_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pP_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pP_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pP_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pP_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pP_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pP_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pP_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pP_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pP_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pP_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pP_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pP_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pP_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pPa_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pPa_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pPa_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pPa_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pPa_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pPa_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pPa_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pPa_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pPa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pPa_times_P(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pPa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pPa_times_Pa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pPa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pPa_times_pP(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_veqm_pPa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_veqm_pPa_times_pPa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_FN_P_xeq_M_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_M_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_M_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_M_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_M_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_M_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_M_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_M_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_Ma_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_Ma_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_Ma_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_Ma_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_Ma_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_Ma_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_Ma_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_Ma_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pM_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pM_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pM_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pM_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pM_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pM_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pM_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pM_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pMa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pMa_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pMa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pMa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pMa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pMa_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pMa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pMa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_P_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_P_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_P_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_P_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_P_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_P_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_P_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_P_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_P_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_P_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_P_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_P_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_P_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_P_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_P_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_P_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_Pa_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_Pa_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_Pa_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_Pa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_Pa_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_Pa_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_Pa_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_Pa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_Pa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_Pa_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_Pa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_Pa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_Pa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_Pa_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_Pa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_Pa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pP_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pP_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pP_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pP_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pP_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pP_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pP_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pP_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pP_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pP_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pP_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pP_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pP_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pP_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pP_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pP_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pPa_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pPa_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pPa_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pPa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pPa_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pPa_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pPa_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pPa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pPa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pPa_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pPa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pPa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pPa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pPa_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeq_pPa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeq_pPa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_M_xeq_spintrace_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_M_xeq_spintrace_P(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_M_xeq_spintrace_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_M_xeq_spintrace_pP(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_FN_P_xpeq_M_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_M_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_M_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_M_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_M_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_M_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_M_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_M_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_Ma_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_Ma_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_Ma_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_Ma_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_Ma_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_Ma_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_Ma_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_Ma_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pM_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pM_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pM_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pM_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pM_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pM_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pM_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pM_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pMa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pMa_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pMa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pMa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pMa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pMa_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pMa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pMa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_P_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_P_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_P_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_P_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_P_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_P_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_P_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_P_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_P_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_P_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_P_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_P_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_P_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_P_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_P_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_P_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_Pa_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_Pa_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_Pa_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_Pa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_Pa_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_Pa_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_Pa_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_Pa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_Pa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_Pa_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_Pa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_Pa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_Pa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_Pa_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_Pa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_Pa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pP_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pP_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pP_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pP_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pP_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pP_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pP_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pP_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pP_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pP_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pP_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pP_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pP_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pP_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pP_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pP_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pPa_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pPa_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pPa_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pPa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pPa_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pPa_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pPa_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pPa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pPa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pPa_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pPa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pPa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pPa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pPa_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xpeq_pPa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xpeq_pPa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_M_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_M_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_M_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_M_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_M_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_M_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_M_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_M_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_Ma_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_Ma_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_Ma_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_Ma_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_Ma_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_Ma_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_Ma_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_Ma_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pM_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pM_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pM_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pM_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pM_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pM_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pM_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pM_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pMa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pMa_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pMa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pMa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pMa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pMa_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pMa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pMa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_P_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_P_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_P_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_P_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_P_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_P_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_P_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_P_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_P_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_P_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_P_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_P_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_P_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_P_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_P_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_P_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_Pa_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_Pa_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_Pa_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_Pa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_Pa_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_Pa_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_Pa_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_Pa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_Pa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_Pa_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_Pa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_Pa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_Pa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_Pa_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_Pa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_Pa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pP_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pP_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pP_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pP_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pP_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pP_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pP_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pP_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pP_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pP_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pP_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pP_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pP_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pP_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pP_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pP_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pPa_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pPa_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pPa_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pPa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pPa_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pPa_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pPa_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pPa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pPa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pPa_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pPa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pPa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pPa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pPa_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xmeq_pPa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xmeq_pPa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_M_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_M_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_M_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_M_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_M_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_M_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_M_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_M_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_Ma_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_Ma_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_Ma_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_Ma_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_Ma_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_Ma_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_Ma_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_Ma_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pM_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pM_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pM_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pM_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pM_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pM_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pM_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pM_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pMa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pMa_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pMa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pMa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pMa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pMa_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pMa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pMa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_P_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_P_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_P_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_P_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_P_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_P_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_P_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_P_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_P_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_P_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_P_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_P_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_P_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_P_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_P_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_P_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_Pa_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_Pa_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_Pa_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_Pa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_Pa_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_Pa_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_Pa_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_Pa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_Pa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_Pa_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_Pa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_Pa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_Pa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_Pa_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_Pa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_Pa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pP_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pP_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pP_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pP_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pP_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pP_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pP_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pP_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pP_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pP_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pP_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pP_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pP_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pP_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pP_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pP_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pPa_times_M (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pPa_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pPa_times_Ma (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pPa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pPa_times_pM (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pPa_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pPa_times_pMa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pPa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pPa_times_P (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pPa_times_P(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pPa_times_Pa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pPa_times_Pa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pPa_times_pP (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pPa_times_pP(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_FN_P_xeqm_pPa_times_pPa (lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)) */
void QLA_FN_P_xeqm_pPa_times_pPa(int nc, void * r, void * a, void * b, int * index, int n);
/* ---- multi: replaces the FN functions emitted by lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d) */
/* replaces QLA_FN_V_veq_nM_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_veq_nM_times_nV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_veq_nM_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_veq_nM_times_npV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_veq_nMa_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_veq_nMa_times_nV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_veq_nMa_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_veq_nMa_times_npV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_veq_npM_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_veq_npM_times_nV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_veq_npM_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_veq_npM_times_npV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_veq_npMa_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_veq_npMa_times_nV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_veq_npMa_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_veq_npMa_times_npV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_vpeq_nM_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_vpeq_nM_times_nV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_vpeq_nM_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_vpeq_nM_times_npV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_vpeq_nMa_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_vpeq_nMa_times_nV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_vpeq_nMa_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_vpeq_nMa_times_npV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_vpeq_npM_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_vpeq_npM_times_nV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_vpeq_npM_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_vpeq_npM_times_npV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_vpeq_npMa_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_vpeq_npMa_times_nV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_vpeq_npMa_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_vpeq_npMa_times_npV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_vmeq_nM_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_vmeq_nM_times_nV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_vmeq_nM_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_vmeq_nM_times_npV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_vmeq_nMa_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_vmeq_nMa_times_nV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_vmeq_nMa_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_vmeq_nMa_times_npV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_vmeq_npM_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_vmeq_npM_times_nV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_vmeq_npM_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_vmeq_npM_times_npV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_vmeq_npMa_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_vmeq_npMa_times_nV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_vmeq_npMa_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_vmeq_npMa_times_npV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_veqm_nM_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_veqm_nM_times_nV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_veqm_nM_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_veqm_nM_times_npV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_veqm_nMa_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_veqm_nMa_times_nV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_veqm_nMa_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_veqm_nMa_times_npV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_veqm_npM_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_veqm_npM_times_nV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_veqm_npM_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_veqm_npM_times_npV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_veqm_npMa_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_veqm_npMa_times_nV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_veqm_npMa_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_veqm_npMa_times_npV(int nc, void * r, void * a, void * b, int n, int nd);
/* replaces QLA_FN_V_xeq_nM_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xeq_nM_times_nV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xeq_nM_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xeq_nM_times_npV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xeq_nMa_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xeq_nMa_times_nV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xeq_nMa_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xeq_nMa_times_npV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xeq_npM_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xeq_npM_times_nV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xeq_npM_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xeq_npM_times_npV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xeq_npMa_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xeq_npMa_times_nV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xeq_npMa_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xeq_npMa_times_npV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xpeq_nM_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xpeq_nM_times_nV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xpeq_nM_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xpeq_nM_times_npV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xpeq_nMa_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xpeq_nMa_times_nV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xpeq_nMa_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xpeq_nMa_times_npV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xpeq_npM_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xpeq_npM_times_nV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xpeq_npM_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xpeq_npM_times_npV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xpeq_npMa_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xpeq_npMa_times_nV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xpeq_npMa_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xpeq_npMa_times_npV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xmeq_nM_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xmeq_nM_times_nV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xmeq_nM_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xmeq_nM_times_npV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xmeq_nMa_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xmeq_nMa_times_nV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xmeq_nMa_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xmeq_nMa_times_npV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xmeq_npM_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xmeq_npM_times_nV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xmeq_npM_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xmeq_npM_times_npV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xmeq_npMa_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xmeq_npMa_times_nV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xmeq_npMa_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xmeq_npMa_times_npV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xeqm_nM_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xeqm_nM_times_nV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xeqm_nM_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xeqm_nM_times_npV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xeqm_nMa_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xeqm_nMa_times_nV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xeqm_nMa_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xeqm_nMa_times_npV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xeqm_npM_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xeqm_npM_times_nV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xeqm_npM_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xeqm_npM_times_npV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xeqm_npMa_times_nV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xeqm_npMa_times_nV(int nc, void * r, void * a, void * b, int * index, int n, int nd);
/* replaces QLA_FN_V_xeqm_npMa_times_npV (lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)) */
void QLA_FN_V_xeqm_npMa_times_npV(int nc, void * r, void * a, void * b, int * index, int n, int nd);

#ifdef __cplusplus
}
#endif
#endif
