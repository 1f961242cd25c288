/*
 * qla_b200_dn.h -- GENERATED by qla_b200/gen/gen_qla.py; do not edit.
 *
 * QLA DN level-1 entry points implemented by libqla_b200.so (sm_100a).
 * Each declaration replaces the reference function of the same name, whose
 * C loop the reference generator emits from the cited section.  Array
 * arguments are device pointers; see qla_b200_runtime.h for scalars,
 * reduction outputs, streams and errors.
 */
#ifndef QLA_B200_DN_H
#define QLA_B200_DN_H
#include "qla_b200_types.h"

#ifdef __cplusplus
#define QLA_B200_RESTRICT __restrict__
extern "C" {
#else
#define QLA_B200_RESTRICT restrict
#endif

/* ---- lmult: replaces the DN functions emitted by lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix) */
/* replaces QLA_DN_V_veq_M_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_veq_M_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_veq_M_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_veq_M_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_veq_Ma_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_veq_Ma_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_veq_Ma_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_veq_Ma_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_veq_pM_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_veq_pM_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_veq_pM_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_veq_pM_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_veq_pMa_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_veq_pMa_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_veq_pMa_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_veq_pMa_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_vpeq_M_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_vpeq_M_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_vpeq_M_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_vpeq_M_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_vpeq_Ma_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_vpeq_Ma_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_vpeq_Ma_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_vpeq_Ma_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_vpeq_pM_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_vpeq_pM_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_vpeq_pM_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_vpeq_pM_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_vpeq_pMa_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_vpeq_pMa_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_vpeq_pMa_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_vpeq_pMa_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_vmeq_M_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_vmeq_M_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_vmeq_M_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_vmeq_M_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_vmeq_Ma_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_vmeq_Ma_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_vmeq_Ma_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_vmeq_Ma_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_vmeq_pM_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_vmeq_pM_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_vmeq_pM_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_vmeq_pM_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_vmeq_pMa_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_vmeq_pMa_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_vmeq_pMa_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_vmeq_pMa_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_veqm_M_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_veqm_M_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_veqm_M_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_veqm_M_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_veqm_Ma_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_veqm_Ma_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_veqm_Ma_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_veqm_Ma_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_veqm_pM_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_veqm_pM_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_veqm_pM_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_veqm_pM_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_veqm_pMa_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_veqm_pMa_times_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_veqm_pMa_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_veqm_pMa_times_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_xeq_M_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xeq_M_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xeq_M_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xeq_M_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xeq_Ma_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xeq_Ma_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xeq_Ma_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xeq_Ma_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xeq_pM_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xeq_pM_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xeq_pM_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xeq_pM_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xeq_pMa_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xeq_pMa_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xeq_pMa_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xeq_pMa_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xpeq_M_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xpeq_M_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xpeq_M_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xpeq_M_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xpeq_Ma_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xpeq_Ma_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xpeq_Ma_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xpeq_Ma_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xpeq_pM_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xpeq_pM_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xpeq_pM_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xpeq_pM_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xpeq_pMa_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xpeq_pMa_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xpeq_pMa_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xpeq_pMa_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xmeq_M_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xmeq_M_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xmeq_M_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xmeq_M_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xmeq_Ma_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xmeq_Ma_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xmeq_Ma_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xmeq_Ma_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xmeq_pM_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xmeq_pM_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xmeq_pM_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xmeq_pM_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xmeq_pMa_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xmeq_pMa_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xmeq_pMa_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xmeq_pMa_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xeqm_M_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xeqm_M_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xeqm_M_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xeqm_M_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xeqm_Ma_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xeqm_Ma_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xeqm_Ma_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xeqm_Ma_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xeqm_pM_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xeqm_pM_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xeqm_pM_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xeqm_pM_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xeqm_pMa_times_V (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xeqm_pMa_times_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xeqm_pMa_times_pV (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_V_xeqm_pMa_times_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_eq_M_times_xV (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_V_eq_M_times_xV(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_V_eq_Ma_times_xV (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_V_eq_Ma_times_xV(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_V_peq_M_times_xV (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_V_peq_M_times_xV(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_V_peq_Ma_times_xV (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_V_peq_Ma_times_xV(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_V_meq_M_times_xV (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_V_meq_M_times_xV(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_V_meq_Ma_times_xV (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_V_meq_Ma_times_xV(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_V_eqm_M_times_xV (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_V_eqm_M_times_xV(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_V_eqm_Ma_times_xV (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_V_eqm_Ma_times_xV(int nc, void * r, void * a, void * b, int * jb, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_V_veq_r_times_V (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_V_veq_r_times_V(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_V_veq_V (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_V_veq_V(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_V_veq_r_times_pV (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_V_veq_r_times_pV(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_V_veq_pV (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_V_veq_pV(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_V_vpeq_r_times_V (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_V_vpeq_r_times_V(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_V_vpeq_V (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_V_vpeq_V(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_V_vpeq_r_times_pV (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_V_vpeq_r_times_pV(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_V_vpeq_pV (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_V_vpeq_pV(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_V_vmeq_r_times_V (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_V_vmeq_r_times_V(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_V_vmeq_V (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_V_vmeq_V(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_V_vmeq_r_times_pV (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_V_vmeq_r_times_pV(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_V_vmeq_pV (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_V_vmeq_pV(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_V_veqm_r_times_V (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_V_veqm_r_times_V(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_V_veqm_V (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_V_veqm_V(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_V_veqm_r_times_pV (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_V_veqm_r_times_pV(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_V_veqm_pV (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_V_veqm_pV(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_V_xeq_r_times_V (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_V_xeq_r_times_V(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_V_xeq_V (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_V_xeq_V(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_V_xeq_r_times_pV (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_V_xeq_r_times_pV(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_V_xeq_pV (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_V_xeq_pV(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_V_xpeq_r_times_V (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_V_xpeq_r_times_V(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_V_xpeq_V (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_V_xpeq_V(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_V_xpeq_r_times_pV (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_V_xpeq_r_times_pV(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_V_xpeq_pV (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_V_xpeq_pV(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_V_xmeq_r_times_V (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_V_xmeq_r_times_V(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_V_xmeq_V (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_V_xmeq_V(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_V_xmeq_r_times_pV (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_V_xmeq_r_times_pV(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_V_xmeq_pV (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_V_xmeq_pV(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_V_xeqm_r_times_V (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_V_xeqm_r_times_V(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_V_xeqm_V (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_V_xeqm_V(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_V_xeqm_r_times_pV (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_V_xeqm_r_times_pV(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_V_xeqm_pV (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_V_xeqm_pV(int nc, void * r, void * a, int * index, int n);
/* ---- norm2: replaces the DN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DN_r_veq_norm2_V (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DN_r_veq_norm2_V(int nc, QLA_D_Real * r, void * a, int n);
/* replaces QLA_DN_r_veq_norm2_pV (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DN_r_veq_norm2_pV(int nc, QLA_D_Real * r, void * a, int n);
/* ---- dot: replaces the DN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DN_c_veq_V_dot_V (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_veq_V_dot_V(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DN_c_veq_V_dot_pV (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_veq_V_dot_pV(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DN_c_veq_pV_dot_V (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_veq_pV_dot_V(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DN_c_veq_pV_dot_pV (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_veq_pV_dot_pV(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* ---- norm2: replaces the DN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DN_r_xeq_norm2_V (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DN_r_xeq_norm2_V(int nc, QLA_D_Real * r, void * a, int * index, int n);
/* replaces QLA_DN_r_xeq_norm2_pV (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DN_r_xeq_norm2_pV(int nc, QLA_D_Real * r, void * a, int * index, int n);
/* ---- dot: replaces the DN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DN_c_xeq_V_dot_V (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_xeq_V_dot_V(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_c_xeq_V_dot_pV (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_xeq_V_dot_pV(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_c_xeq_pV_dot_V (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_xeq_pV_dot_V(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_c_xeq_pV_dot_pV (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_xeq_pV_dot_pV(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* ---- lmult: replaces the DN functions emitted by lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix) */
/* replaces QLA_DN_H_veq_M_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_veq_M_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_veq_M_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_veq_M_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_veq_Ma_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_veq_Ma_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_veq_Ma_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_veq_Ma_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_veq_pM_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_veq_pM_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_veq_pM_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_veq_pM_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_veq_pMa_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_veq_pMa_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_veq_pMa_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_veq_pMa_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_vpeq_M_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_vpeq_M_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_vpeq_M_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_vpeq_M_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_vpeq_Ma_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_vpeq_Ma_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_vpeq_Ma_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_vpeq_Ma_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_vpeq_pM_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_vpeq_pM_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_vpeq_pM_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_vpeq_pM_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_vpeq_pMa_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_vpeq_pMa_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_vpeq_pMa_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_vpeq_pMa_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_vmeq_M_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_vmeq_M_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_vmeq_M_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_vmeq_M_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_vmeq_Ma_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_vmeq_Ma_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_vmeq_Ma_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_vmeq_Ma_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_vmeq_pM_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_vmeq_pM_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_vmeq_pM_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_vmeq_pM_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_vmeq_pMa_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_vmeq_pMa_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_vmeq_pMa_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_vmeq_pMa_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_veqm_M_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_veqm_M_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_veqm_M_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_veqm_M_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_veqm_Ma_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_veqm_Ma_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_veqm_Ma_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_veqm_Ma_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_veqm_pM_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_veqm_pM_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_veqm_pM_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_veqm_pM_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_veqm_pMa_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_veqm_pMa_times_H(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_veqm_pMa_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_veqm_pMa_times_pH(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_H_xeq_M_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xeq_M_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xeq_M_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xeq_M_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xeq_Ma_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xeq_Ma_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xeq_Ma_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xeq_Ma_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xeq_pM_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xeq_pM_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xeq_pM_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xeq_pM_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xeq_pMa_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xeq_pMa_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xeq_pMa_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xeq_pMa_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xpeq_M_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xpeq_M_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xpeq_M_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xpeq_M_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xpeq_Ma_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xpeq_Ma_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xpeq_Ma_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xpeq_Ma_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xpeq_pM_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xpeq_pM_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xpeq_pM_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xpeq_pM_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xpeq_pMa_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xpeq_pMa_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xpeq_pMa_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xpeq_pMa_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xmeq_M_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xmeq_M_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xmeq_M_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xmeq_M_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xmeq_Ma_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xmeq_Ma_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xmeq_Ma_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xmeq_Ma_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xmeq_pM_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xmeq_pM_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xmeq_pM_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xmeq_pM_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xmeq_pMa_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xmeq_pMa_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xmeq_pMa_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xmeq_pMa_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xeqm_M_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xeqm_M_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xeqm_M_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xeqm_M_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xeqm_Ma_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xeqm_Ma_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xeqm_Ma_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xeqm_Ma_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xeqm_pM_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xeqm_pM_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xeqm_pM_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xeqm_pM_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xeqm_pMa_times_H (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xeqm_pMa_times_H(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_xeqm_pMa_times_pH (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_H_xeqm_pMa_times_pH(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_H_eq_M_times_xH (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_H_eq_M_times_xH(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_H_eq_Ma_times_xH (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_H_eq_Ma_times_xH(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_H_peq_M_times_xH (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_H_peq_M_times_xH(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_H_peq_Ma_times_xH (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_H_peq_Ma_times_xH(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_H_meq_M_times_xH (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_H_meq_M_times_xH(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_H_meq_Ma_times_xH (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_H_meq_Ma_times_xH(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_H_eqm_M_times_xH (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_H_eqm_M_times_xH(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_H_eqm_Ma_times_xH (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_H_eqm_Ma_times_xH(int nc, void * r, void * a, void * b, int * jb, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_H_veq_r_times_H (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_H_veq_r_times_H(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_H_veq_H (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_H_veq_H(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_H_veq_r_times_pH (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_H_veq_r_times_pH(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_H_veq_pH (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_H_veq_pH(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_H_vpeq_r_times_H (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_H_vpeq_r_times_H(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_H_vpeq_H (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_H_vpeq_H(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_H_vpeq_r_times_pH (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_H_vpeq_r_times_pH(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_H_vpeq_pH (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_H_vpeq_pH(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_H_vmeq_r_times_H (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_H_vmeq_r_times_H(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_H_vmeq_H (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_H_vmeq_H(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_H_vmeq_r_times_pH (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_H_vmeq_r_times_pH(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_H_vmeq_pH (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_H_vmeq_pH(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_H_veqm_r_times_H (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_H_veqm_r_times_H(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_H_veqm_H (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_H_veqm_H(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_H_veqm_r_times_pH (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_H_veqm_r_times_pH(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_H_veqm_pH (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_H_veqm_pH(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_H_xeq_r_times_H (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_H_xeq_r_times_H(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_H_xeq_H (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_H_xeq_H(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_H_xeq_r_times_pH (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_H_xeq_r_times_pH(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_H_xeq_pH (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_H_xeq_pH(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_H_xpeq_r_times_H (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_H_xpeq_r_times_H(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_H_xpeq_H (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_H_xpeq_H(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_H_xpeq_r_times_pH (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_H_xpeq_r_times_pH(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_H_xpeq_pH (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_H_xpeq_pH(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_H_xmeq_r_times_H (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_H_xmeq_r_times_H(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_H_xmeq_H (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_H_xmeq_H(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_H_xmeq_r_times_pH (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_H_xmeq_r_times_pH(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_H_xmeq_pH (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_H_xmeq_pH(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_H_xeqm_r_times_H (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_H_xeqm_r_times_H(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_H_xeqm_H (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_H_xeqm_H(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_H_xeqm_r_times_pH (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_H_xeqm_r_times_pH(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_H_xeqm_pH (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_H_xeqm_pH(int nc, void * r, void * a, int * index, int n);
/* ---- norm2: replaces the DN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DN_r_veq_norm2_H (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DN_r_veq_norm2_H(int nc, QLA_D_Real * r, void * a, int n);
/* replaces QLA_DN_r_veq_norm2_pH (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DN_r_veq_norm2_pH(int nc, QLA_D_Real * r, void * a, int n);
/* ---- dot: replaces the DN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DN_c_veq_H_dot_H (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_veq_H_dot_H(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DN_c_veq_H_dot_pH (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_veq_H_dot_pH(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DN_c_veq_pH_dot_H (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_veq_pH_dot_H(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DN_c_veq_pH_dot_pH (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_veq_pH_dot_pH(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* ---- norm2: replaces the DN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DN_r_xeq_norm2_H (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DN_r_xeq_norm2_H(int nc, QLA_D_Real * r, void * a, int * index, int n);
/* replaces QLA_DN_r_xeq_norm2_pH (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DN_r_xeq_norm2_pH(int nc, QLA_D_Real * r, void * a, int * index, int n);
/* ---- dot: replaces the DN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DN_c_xeq_H_dot_H (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_xeq_H_dot_H(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_c_xeq_H_dot_pH (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_xeq_H_dot_pH(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_c_xeq_pH_dot_H (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_xeq_pH_dot_H(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_c_xeq_pH_dot_pH (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_xeq_pH_dot_pH(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* ---- lmult: replaces the DN functions emitted by lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix) */
/* replaces QLA_DN_D_veq_M_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_veq_M_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_veq_M_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_veq_M_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_veq_Ma_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_veq_Ma_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_veq_Ma_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_veq_Ma_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_veq_pM_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_veq_pM_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_veq_pM_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_veq_pM_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_veq_pMa_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_veq_pMa_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_veq_pMa_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_veq_pMa_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_vpeq_M_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_vpeq_M_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_vpeq_M_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_vpeq_M_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_vpeq_Ma_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_vpeq_Ma_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_vpeq_Ma_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_vpeq_Ma_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_vpeq_pM_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_vpeq_pM_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_vpeq_pM_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_vpeq_pM_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_vpeq_pMa_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_vpeq_pMa_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_vpeq_pMa_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_vpeq_pMa_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_vmeq_M_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_vmeq_M_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_vmeq_M_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_vmeq_M_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_vmeq_Ma_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_vmeq_Ma_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_vmeq_Ma_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_vmeq_Ma_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_vmeq_pM_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_vmeq_pM_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_vmeq_pM_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_vmeq_pM_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_vmeq_pMa_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_vmeq_pMa_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_vmeq_pMa_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_vmeq_pMa_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_veqm_M_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_veqm_M_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_veqm_M_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_veqm_M_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_veqm_Ma_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_veqm_Ma_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_veqm_Ma_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_veqm_Ma_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_veqm_pM_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_veqm_pM_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_veqm_pM_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_veqm_pM_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_veqm_pMa_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_veqm_pMa_times_D(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_veqm_pMa_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_veqm_pMa_times_pD(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_D_xeq_M_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xeq_M_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xeq_M_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xeq_M_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xeq_Ma_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xeq_Ma_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xeq_Ma_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xeq_Ma_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xeq_pM_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xeq_pM_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xeq_pM_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xeq_pM_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xeq_pMa_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xeq_pMa_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xeq_pMa_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xeq_pMa_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xpeq_M_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xpeq_M_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xpeq_M_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xpeq_M_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xpeq_Ma_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xpeq_Ma_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xpeq_Ma_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xpeq_Ma_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xpeq_pM_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xpeq_pM_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xpeq_pM_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xpeq_pM_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xpeq_pMa_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xpeq_pMa_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xpeq_pMa_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xpeq_pMa_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xmeq_M_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xmeq_M_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xmeq_M_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xmeq_M_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xmeq_Ma_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xmeq_Ma_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xmeq_Ma_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xmeq_Ma_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xmeq_pM_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xmeq_pM_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xmeq_pM_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xmeq_pM_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xmeq_pMa_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xmeq_pMa_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xmeq_pMa_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xmeq_pMa_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xeqm_M_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xeqm_M_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xeqm_M_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xeqm_M_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xeqm_Ma_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xeqm_Ma_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xeqm_Ma_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xeqm_Ma_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xeqm_pM_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xeqm_pM_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xeqm_pM_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xeqm_pM_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xeqm_pMa_times_D (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xeqm_pMa_times_D(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_xeqm_pMa_times_pD (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_D_xeqm_pMa_times_pD(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_D_eq_M_times_xD (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_D_eq_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_D_eq_Ma_times_xD (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_D_eq_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_D_peq_M_times_xD (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_D_peq_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_D_peq_Ma_times_xD (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_D_peq_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_D_meq_M_times_xD (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_D_meq_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_D_meq_Ma_times_xD (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_D_meq_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_D_eqm_M_times_xD (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_D_eqm_M_times_xD(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_D_eqm_Ma_times_xD (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_D_eqm_Ma_times_xD(int nc, void * r, void * a, void * b, int * jb, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_D_veq_r_times_D (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_D_veq_r_times_D(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_D_veq_D (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_D_veq_D(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_D_veq_r_times_pD (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_D_veq_r_times_pD(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_D_veq_pD (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_D_veq_pD(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_D_vpeq_r_times_D (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_D_vpeq_r_times_D(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_D_vpeq_D (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_D_vpeq_D(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_D_vpeq_r_times_pD (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_D_vpeq_r_times_pD(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_D_vpeq_pD (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_D_vpeq_pD(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_D_vmeq_r_times_D (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_D_vmeq_r_times_D(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_D_vmeq_D (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_D_vmeq_D(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_D_vmeq_r_times_pD (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_D_vmeq_r_times_pD(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_D_vmeq_pD (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_D_vmeq_pD(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_D_veqm_r_times_D (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_D_veqm_r_times_D(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_D_veqm_D (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_D_veqm_D(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_D_veqm_r_times_pD (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_D_veqm_r_times_pD(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_D_veqm_pD (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_D_veqm_pD(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_D_xeq_r_times_D (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_D_xeq_r_times_D(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_D_xeq_D (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_D_xeq_D(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_D_xeq_r_times_pD (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_D_xeq_r_times_pD(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_D_xeq_pD (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_D_xeq_pD(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_D_xpeq_r_times_D (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_D_xpeq_r_times_D(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_D_xpeq_D (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_D_xpeq_D(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_D_xpeq_r_times_pD (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_D_xpeq_r_times_pD(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_D_xpeq_pD (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_D_xpeq_pD(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_D_xmeq_r_times_D (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_D_xmeq_r_times_D(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_D_xmeq_D (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_D_xmeq_D(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_D_xmeq_r_times_pD (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_D_xmeq_r_times_pD(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_D_xmeq_pD (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_D_xmeq_pD(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_D_xeqm_r_times_D (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_D_xeqm_r_times_D(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_D_xeqm_D (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_D_xeqm_D(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_D_xeqm_r_times_pD (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_D_xeqm_r_times_pD(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_D_xeqm_pD (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_D_xeqm_pD(int nc, void * r, void * a, int * index, int n);
/* ---- norm2: replaces the DN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DN_r_veq_norm2_D (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DN_r_veq_norm2_D(int nc, QLA_D_Real * r, void * a, int n);
/* replaces QLA_DN_r_veq_norm2_pD (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DN_r_veq_norm2_pD(int nc, QLA_D_Real * r, void * a, int n);
/* ---- dot: replaces the DN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DN_c_veq_D_dot_D (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_veq_D_dot_D(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DN_c_veq_D_dot_pD (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_veq_D_dot_pD(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DN_c_veq_pD_dot_D (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_veq_pD_dot_D(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DN_c_veq_pD_dot_pD (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_veq_pD_dot_pD(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* ---- norm2: replaces the DN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DN_r_xeq_norm2_D (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DN_r_xeq_norm2_D(int nc, QLA_D_Real * r, void * a, int * index, int n);
/* replaces QLA_DN_r_xeq_norm2_pD (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DN_r_xeq_norm2_pD(int nc, QLA_D_Real * r, void * a, int * index, int n);
/* ---- dot: replaces the DN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DN_c_xeq_D_dot_D (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_xeq_D_dot_D(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_c_xeq_D_dot_pD (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_xeq_D_dot_pD(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_c_xeq_pD_dot_D (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_xeq_pD_dot_D(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_c_xeq_pD_dot_pD (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_xeq_pD_dot_pD(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* ---- lmult: replaces the DN functions emitted by lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix) */
/* replaces QLA_DN_M_veq_M_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veq_M_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veq_M_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veq_M_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veq_M_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veq_M_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veq_M_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veq_M_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veq_Ma_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veq_Ma_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veq_Ma_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veq_Ma_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veq_Ma_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veq_Ma_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veq_Ma_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veq_Ma_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veq_pM_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veq_pM_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veq_pM_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veq_pM_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veq_pM_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veq_pM_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veq_pM_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veq_pM_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veq_pMa_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veq_pMa_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veq_pMa_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veq_pMa_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veq_pMa_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veq_pMa_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veq_pMa_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veq_pMa_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vpeq_M_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vpeq_M_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vpeq_M_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vpeq_M_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vpeq_M_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vpeq_M_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vpeq_M_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vpeq_M_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vpeq_Ma_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vpeq_Ma_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vpeq_Ma_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vpeq_Ma_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vpeq_Ma_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vpeq_Ma_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vpeq_Ma_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vpeq_Ma_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vpeq_pM_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vpeq_pM_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vpeq_pM_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vpeq_pM_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vpeq_pM_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vpeq_pM_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vpeq_pM_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vpeq_pM_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vpeq_pMa_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vpeq_pMa_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vpeq_pMa_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vpeq_pMa_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vpeq_pMa_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vpeq_pMa_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vpeq_pMa_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vpeq_pMa_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vmeq_M_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vmeq_M_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vmeq_M_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vmeq_M_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vmeq_M_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vmeq_M_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vmeq_M_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vmeq_M_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vmeq_Ma_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vmeq_Ma_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vmeq_Ma_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vmeq_Ma_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vmeq_Ma_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vmeq_Ma_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vmeq_Ma_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vmeq_Ma_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vmeq_pM_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vmeq_pM_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vmeq_pM_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vmeq_pM_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vmeq_pM_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vmeq_pM_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vmeq_pM_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vmeq_pM_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vmeq_pMa_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vmeq_pMa_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vmeq_pMa_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vmeq_pMa_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vmeq_pMa_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vmeq_pMa_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_vmeq_pMa_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_vmeq_pMa_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veqm_M_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veqm_M_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veqm_M_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veqm_M_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veqm_M_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veqm_M_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veqm_M_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veqm_M_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veqm_Ma_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veqm_Ma_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veqm_Ma_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veqm_Ma_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veqm_Ma_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veqm_Ma_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veqm_Ma_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veqm_Ma_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veqm_pM_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veqm_pM_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veqm_pM_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veqm_pM_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veqm_pM_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veqm_pM_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veqm_pM_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veqm_pM_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veqm_pMa_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veqm_pMa_times_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veqm_pMa_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veqm_pMa_times_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veqm_pMa_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veqm_pMa_times_Ma(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veqm_pMa_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_veqm_pMa_times_pMa(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_xeq_M_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeq_M_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeq_M_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeq_M_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeq_M_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeq_M_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeq_M_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeq_M_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeq_Ma_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeq_Ma_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeq_Ma_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeq_Ma_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeq_Ma_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeq_Ma_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeq_Ma_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeq_Ma_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeq_pM_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeq_pM_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeq_pM_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeq_pM_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeq_pM_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeq_pM_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeq_pM_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeq_pM_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeq_pMa_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeq_pMa_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeq_pMa_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeq_pMa_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeq_pMa_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeq_pMa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeq_pMa_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeq_pMa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xpeq_M_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xpeq_M_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xpeq_M_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xpeq_M_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xpeq_M_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xpeq_M_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xpeq_M_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xpeq_M_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xpeq_Ma_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xpeq_Ma_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xpeq_Ma_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xpeq_Ma_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xpeq_Ma_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xpeq_Ma_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xpeq_Ma_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xpeq_Ma_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xpeq_pM_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xpeq_pM_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xpeq_pM_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xpeq_pM_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xpeq_pM_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xpeq_pM_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xpeq_pM_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xpeq_pM_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xpeq_pMa_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xpeq_pMa_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xpeq_pMa_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xpeq_pMa_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xpeq_pMa_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xpeq_pMa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xpeq_pMa_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xpeq_pMa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xmeq_M_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xmeq_M_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xmeq_M_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xmeq_M_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xmeq_M_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xmeq_M_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xmeq_M_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xmeq_M_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xmeq_Ma_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xmeq_Ma_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xmeq_Ma_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xmeq_Ma_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xmeq_Ma_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xmeq_Ma_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xmeq_Ma_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xmeq_Ma_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xmeq_pM_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xmeq_pM_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xmeq_pM_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xmeq_pM_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xmeq_pM_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xmeq_pM_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xmeq_pM_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xmeq_pM_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xmeq_pMa_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xmeq_pMa_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xmeq_pMa_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xmeq_pMa_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xmeq_pMa_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xmeq_pMa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xmeq_pMa_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xmeq_pMa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeqm_M_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeqm_M_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeqm_M_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeqm_M_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeqm_M_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeqm_M_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeqm_M_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeqm_M_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeqm_Ma_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeqm_Ma_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeqm_Ma_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeqm_Ma_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeqm_Ma_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeqm_Ma_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeqm_Ma_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeqm_Ma_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeqm_pM_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeqm_pM_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeqm_pM_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeqm_pM_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeqm_pM_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeqm_pM_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeqm_pM_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeqm_pM_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeqm_pMa_times_M (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeqm_pMa_times_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeqm_pMa_times_pM (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeqm_pMa_times_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeqm_pMa_times_Ma (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeqm_pMa_times_Ma(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeqm_pMa_times_pMa (lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766) */
void QLA_DN_M_xeqm_pMa_times_pMa(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_eq_M_times_xM (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_M_eq_M_times_xM(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_M_eq_Ma_times_xM (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_M_eq_Ma_times_xM(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_M_peq_M_times_xM (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_M_peq_M_times_xM(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_M_peq_Ma_times_xM (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_M_peq_Ma_times_xM(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_M_meq_M_times_xM (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_M_meq_M_times_xM(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_M_meq_Ma_times_xM (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_M_meq_Ma_times_xM(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_M_eqm_M_times_xM (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_M_eqm_M_times_xM(int nc, void * r, void * a, void * b, int * jb, int n);
/* replaces QLA_DN_M_eqm_Ma_times_xM (doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)) */
void QLA_DN_M_eqm_Ma_times_xM(int nc, void * r, void * a, void * b, int * jb, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_M_veq_r_times_M (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_M_veq_r_times_M(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_M_veq_M (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_M_veq_M(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_M_veq_r_times_pM (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_M_veq_r_times_pM(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_M_veq_pM (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_M_veq_pM(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_M_vpeq_r_times_M (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_M_vpeq_r_times_M(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_M_vpeq_M (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_M_vpeq_M(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_M_vpeq_r_times_pM (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_M_vpeq_r_times_pM(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_M_vpeq_pM (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_M_vpeq_pM(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_M_vmeq_r_times_M (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_M_vmeq_r_times_M(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_M_vmeq_M (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_M_vmeq_M(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_M_vmeq_r_times_pM (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_M_vmeq_r_times_pM(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_M_vmeq_pM (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_M_vmeq_pM(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_M_veqm_r_times_M (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_M_veqm_r_times_M(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_M_veqm_M (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_M_veqm_M(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_M_veqm_r_times_pM (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_M_veqm_r_times_pM(int nc, void * r, QLA_D_Real * a, void * b, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_M_veqm_pM (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_M_veqm_pM(int nc, void * r, void * a, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_M_xeq_r_times_M (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_M_xeq_r_times_M(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_M_xeq_M (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_M_xeq_M(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_M_xeq_r_times_pM (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_M_xeq_r_times_pM(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_M_xeq_pM (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_M_xeq_pM(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_M_xpeq_r_times_M (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_M_xpeq_r_times_M(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_M_xpeq_M (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_M_xpeq_M(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_M_xpeq_r_times_pM (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_M_xpeq_r_times_pM(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_M_xpeq_pM (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_M_xpeq_pM(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_M_xmeq_r_times_M (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_M_xmeq_r_times_M(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_M_xmeq_M (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_M_xmeq_M(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_M_xmeq_r_times_pM (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_M_xmeq_r_times_pM(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_M_xmeq_pM (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_M_xmeq_pM(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_M_xeqm_r_times_M (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_M_xeqm_r_times_M(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_M_xeqm_M (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_M_xeqm_M(int nc, void * r, void * a, int * index, int n);
/* ---- rtimes: replaces the DN functions emitted by lib/perl/build_qla.pl:1256-1292 (real constant times field) */
/* replaces QLA_DN_M_xeqm_r_times_pM (lib/perl/build_qla.pl:1256-1292 (real constant times field)) */
void QLA_DN_M_xeqm_r_times_pM(int nc, void * r, QLA_D_Real * a, void * b, int * index, int n);
/* ---- copy: replaces the DN functions emitted by lib/perl/build_qla.pl:370-400 (assignment / gather) */
/* replaces QLA_DN_M_xeqm_pM (lib/perl/build_qla.pl:370-400 (assignment / gather)) */
void QLA_DN_M_xeqm_pM(int nc, void * r, void * a, int * index, int n);
/* ---- norm2: replaces the DN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DN_r_veq_norm2_M (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DN_r_veq_norm2_M(int nc, QLA_D_Real * r, void * a, int n);
/* replaces QLA_DN_r_veq_norm2_pM (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DN_r_veq_norm2_pM(int nc, QLA_D_Real * r, void * a, int n);
/* ---- dot: replaces the DN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DN_c_veq_M_dot_M (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_veq_M_dot_M(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DN_c_veq_M_dot_pM (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_veq_M_dot_pM(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DN_c_veq_pM_dot_M (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_veq_pM_dot_M(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DN_c_veq_pM_dot_pM (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_veq_pM_dot_pM(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* ---- norm2: replaces the DN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DN_r_xeq_norm2_M (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DN_r_xeq_norm2_M(int nc, QLA_D_Real * r, void * a, int * index, int n);
/* replaces QLA_DN_r_xeq_norm2_pM (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DN_r_xeq_norm2_pM(int nc, QLA_D_Real * r, void * a, int * index, int n);
/* ---- dot: replaces the DN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DN_c_xeq_M_dot_M (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_xeq_M_dot_M(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_c_xeq_M_dot_pM (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_xeq_M_dot_pM(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_c_xeq_pM_dot_M (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_xeq_pM_dot_M(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_c_xeq_pM_dot_pM (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DN_c_xeq_pM_dot_pM(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* ---- spproj: replaces the DN functions emitted by lib/perl/build_qla.pl:1087-1110 */
/* replaces QLA_DN_H_veq_spproj_D (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_DN_H_veq_spproj_D(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_DN_H_veq_spproj_pD (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_DN_H_veq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int n);
/* ---- sprecon: replaces the DN functions emitted by lib/perl/build_qla.pl:1112-1135 */
/* replaces QLA_DN_D_veq_sprecon_H (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_DN_D_veq_sprecon_H(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_DN_D_veq_sprecon_pH (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_DN_D_veq_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int n);
/* ---- spproj: replaces the DN functions emitted by lib/perl/build_qla.pl:1087-1110 */
/* replaces QLA_DN_H_vpeq_spproj_D (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_DN_H_vpeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_DN_H_vpeq_spproj_pD (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_DN_H_vpeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int n);
/* ---- sprecon: replaces the DN functions emitted by lib/perl/build_qla.pl:1112-1135 */
/* replaces QLA_DN_D_vpeq_sprecon_H (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_DN_D_vpeq_sprecon_H(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_DN_D_vpeq_sprecon_pH (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_DN_D_vpeq_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int n);
/* ---- spproj: replaces the DN functions emitted by lib/perl/build_qla.pl:1087-1110 */
/* replaces QLA_DN_H_vmeq_spproj_D (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_DN_H_vmeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_DN_H_vmeq_spproj_pD (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_DN_H_vmeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int n);
/* ---- sprecon: replaces the DN functions emitted by lib/perl/build_qla.pl:1112-1135 */
/* replaces QLA_DN_D_vmeq_sprecon_H (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_DN_D_vmeq_sprecon_H(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_DN_D_vmeq_sprecon_pH (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_DN_D_vmeq_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int n);
/* ---- spproj: replaces the DN functions emitted by lib/perl/build_qla.pl:1087-1110 */
/* replaces QLA_DN_H_veqm_spproj_D (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_DN_H_veqm_spproj_D(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_DN_H_veqm_spproj_pD (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_DN_H_veqm_spproj_pD(int nc, void * r, void * a, int mu, int sign, int n);
/* ---- sprecon: replaces the DN functions emitted by lib/perl/build_qla.pl:1112-1135 */
/* replaces QLA_DN_D_veqm_sprecon_H (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_DN_D_veqm_sprecon_H(int nc, void * r, void * a, int mu, int sign, int n);
/* replaces QLA_DN_D_veqm_sprecon_pH (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_DN_D_veqm_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int n);
/* ---- mfunc: replaces the DN functions emitted by lib/perl/build_qla.pl:1000-1060 (matrix functions) */
/* replaces QLA_DN_M_veq_exp_M (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_DN_M_veq_exp_M(int nc, void * r, void * a, int n);
/* replaces QLA_DN_M_veq_sqrt_M (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_DN_M_veq_sqrt_M(int nc, void * r, void * a, int n);
/* replaces QLA_DN_M_veq_inverse_M (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_DN_M_veq_inverse_M(int nc, void * r, void * a, int n);
/* replaces QLA_DN_C_veq_det_M (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_DN_C_veq_det_M(int nc, QLA_D_Complex * r, void * a, int n);
/* ---- mfunc_ext: replaces the DN functions emitted by lib/perl/build_qla.pl:1022-1061 (matrix functions */
/* replaces QLA_DN_M_veq_invsqrt_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_veq_invsqrt_M(int nc, void * r, void * a, int n);
/* replaces QLA_DN_M_veq_log_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_veq_log_M(int nc, void * r, void * a, int n);
/* replaces QLA_DN_M_veq_expA_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_veq_expA_M(int nc, void * r, void * a, int n);
/* replaces QLA_DN_M_veq_expTA_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_veq_expTA_M(int nc, void * r, void * a, int n);
/* replaces QLA_DN_M_veq_sqrtPH_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_veq_sqrtPH_M(int nc, void * r, void * a, int n);
/* replaces QLA_DN_M_veq_invsqrtPH_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_veq_invsqrtPH_M(int nc, void * r, void * a, int n);
/* replaces QLA_DN_V_veq_eigenvals_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_V_veq_eigenvals_M(int nc, void * r, void * a, int n);
/* replaces QLA_DN_V_veq_eigenvalsH_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_V_veq_eigenvalsH_M(int nc, void * r, void * a, int n);
/* ---- mfunc: replaces the DN functions emitted by lib/perl/build_qla.pl:1000-1060 (matrix functions) */
/* replaces QLA_DN_M_veq_exp_pM (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_DN_M_veq_exp_pM(int nc, void * r, void * a, int n);
/* replaces QLA_DN_M_veq_sqrt_pM (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_DN_M_veq_sqrt_pM(int nc, void * r, void * a, int n);
/* replaces QLA_DN_M_veq_inverse_pM (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_DN_M_veq_inverse_pM(int nc, void * r, void * a, int n);
/* replaces QLA_DN_C_veq_det_pM (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_DN_C_veq_det_pM(int nc, QLA_D_Complex * r, void * a, int n);
/* ---- mfunc_ext: replaces the DN functions emitted by lib/perl/build_qla.pl:1022-1061 (matrix functions */
/* replaces QLA_DN_M_veq_invsqrt_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_veq_invsqrt_pM(int nc, void * r, void * a, int n);
/* replaces QLA_DN_M_veq_log_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_veq_log_pM(int nc, void * r, void * a, int n);
/* replaces QLA_DN_M_veq_expA_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_veq_expA_pM(int nc, void * r, void * a, int n);
/* replaces QLA_DN_M_veq_expTA_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_veq_expTA_pM(int nc, void * r, void * a, int n);
/* replaces QLA_DN_M_veq_sqrtPH_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_veq_sqrtPH_pM(int nc, void * r, void * a, int n);
/* replaces QLA_DN_M_veq_invsqrtPH_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_veq_invsqrtPH_pM(int nc, void * r, void * a, int n);
/* replaces QLA_DN_V_veq_eigenvals_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_V_veq_eigenvals_pM(int nc, void * r, void * a, int n);
/* replaces QLA_DN_V_veq_eigenvalsH_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_V_veq_eigenvalsH_pM(int nc, void * r, void * a, int n);
/* replaces QLA_DN_V_veq_M_inverse_V (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_DN_V_veq_M_inverse_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_veq_M_inverse_pV (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_DN_V_veq_M_inverse_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_veq_pM_inverse_V (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_DN_V_veq_pM_inverse_V(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_V_veq_pM_inverse_pV (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_DN_V_veq_pM_inverse_pV(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veq_M_inverse_M (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_DN_M_veq_M_inverse_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veq_M_inverse_pM (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_DN_M_veq_M_inverse_pM(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veq_pM_inverse_M (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_DN_M_veq_pM_inverse_M(int nc, void * r, void * a, void * b, int n);
/* replaces QLA_DN_M_veq_pM_inverse_pM (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_DN_M_veq_pM_inverse_pM(int nc, void * r, void * a, void * b, int n);
/* ---- spproj: replaces the DN functions emitted by lib/perl/build_qla.pl:1087-1110 */
/* replaces QLA_DN_H_xeq_spproj_D (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_DN_H_xeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_DN_H_xeq_spproj_pD (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_DN_H_xeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* ---- sprecon: replaces the DN functions emitted by lib/perl/build_qla.pl:1112-1135 */
/* replaces QLA_DN_D_xeq_sprecon_H (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_DN_D_xeq_sprecon_H(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_DN_D_xeq_sprecon_pH (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_DN_D_xeq_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* ---- spproj: replaces the DN functions emitted by lib/perl/build_qla.pl:1087-1110 */
/* replaces QLA_DN_H_xpeq_spproj_D (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_DN_H_xpeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_DN_H_xpeq_spproj_pD (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_DN_H_xpeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* ---- sprecon: replaces the DN functions emitted by lib/perl/build_qla.pl:1112-1135 */
/* replaces QLA_DN_D_xpeq_sprecon_H (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_DN_D_xpeq_sprecon_H(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_DN_D_xpeq_sprecon_pH (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_DN_D_xpeq_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* ---- spproj: replaces the DN functions emitted by lib/perl/build_qla.pl:1087-1110 */
/* replaces QLA_DN_H_xmeq_spproj_D (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_DN_H_xmeq_spproj_D(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_DN_H_xmeq_spproj_pD (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_DN_H_xmeq_spproj_pD(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* ---- sprecon: replaces the DN functions emitted by lib/perl/build_qla.pl:1112-1135 */
/* replaces QLA_DN_D_xmeq_sprecon_H (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_DN_D_xmeq_sprecon_H(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_DN_D_xmeq_sprecon_pH (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_DN_D_xmeq_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* ---- spproj: replaces the DN functions emitted by lib/perl/build_qla.pl:1087-1110 */
/* replaces QLA_DN_H_xeqm_spproj_D (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_DN_H_xeqm_spproj_D(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_DN_H_xeqm_spproj_pD (lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275) */
void QLA_DN_H_xeqm_spproj_pD(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* ---- sprecon: replaces the DN functions emitted by lib/perl/build_qla.pl:1112-1135 */
/* replaces QLA_DN_D_xeqm_sprecon_H (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_DN_D_xeqm_sprecon_H(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* replaces QLA_DN_D_xeqm_sprecon_pH (lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337) */
void QLA_DN_D_xeqm_sprecon_pH(int nc, void * r, void * a, int mu, int sign, int * index, int n);
/* ---- mfunc: replaces the DN functions emitted by lib/perl/build_qla.pl:1000-1060 (matrix functions) */
/* replaces QLA_DN_M_xeq_exp_M (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_DN_M_xeq_exp_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_DN_M_xeq_sqrt_M (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_DN_M_xeq_sqrt_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_DN_M_xeq_inverse_M (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_DN_M_xeq_inverse_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_DN_C_xeq_det_M (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_DN_C_xeq_det_M(int nc, QLA_D_Complex * r, void * a, int * index, int n);
/* ---- mfunc_ext: replaces the DN functions emitted by lib/perl/build_qla.pl:1022-1061 (matrix functions */
/* replaces QLA_DN_M_xeq_invsqrt_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_xeq_invsqrt_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_DN_M_xeq_log_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_xeq_log_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_DN_M_xeq_expA_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_xeq_expA_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_DN_M_xeq_expTA_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_xeq_expTA_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_DN_M_xeq_sqrtPH_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_xeq_sqrtPH_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_DN_M_xeq_invsqrtPH_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_xeq_invsqrtPH_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_DN_V_xeq_eigenvals_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_V_xeq_eigenvals_M(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_DN_V_xeq_eigenvalsH_M (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_V_xeq_eigenvalsH_M(int nc, void * r, void * a, int * index, int n);
/* ---- mfunc: replaces the DN functions emitted by lib/perl/build_qla.pl:1000-1060 (matrix functions) */
/* replaces QLA_DN_M_xeq_exp_pM (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_DN_M_xeq_exp_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_DN_M_xeq_sqrt_pM (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_DN_M_xeq_sqrt_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_DN_M_xeq_inverse_pM (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_DN_M_xeq_inverse_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_DN_C_xeq_det_pM (lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143) */
void QLA_DN_C_xeq_det_pM(int nc, QLA_D_Complex * r, void * a, int * index, int n);
/* ---- mfunc_ext: replaces the DN functions emitted by lib/perl/build_qla.pl:1022-1061 (matrix functions */
/* replaces QLA_DN_M_xeq_invsqrt_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_xeq_invsqrt_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_DN_M_xeq_log_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_xeq_log_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_DN_M_xeq_expA_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_xeq_expA_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_DN_M_xeq_expTA_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_xeq_expTA_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_DN_M_xeq_sqrtPH_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_xeq_sqrtPH_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_DN_M_xeq_invsqrtPH_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_M_xeq_invsqrtPH_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_DN_V_xeq_eigenvals_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_V_xeq_eigenvals_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_DN_V_xeq_eigenvalsH_pM (lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166) */
void QLA_DN_V_xeq_eigenvalsH_pM(int nc, void * r, void * a, int * index, int n);
/* replaces QLA_DN_V_xeq_M_inverse_V (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_DN_V_xeq_M_inverse_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xeq_M_inverse_pV (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_DN_V_xeq_M_inverse_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xeq_pM_inverse_V (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_DN_V_xeq_pM_inverse_V(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_V_xeq_pM_inverse_pV (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_DN_V_xeq_pM_inverse_pV(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeq_M_inverse_M (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_DN_M_xeq_M_inverse_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeq_M_inverse_pM (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_DN_M_xeq_M_inverse_pM(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeq_pM_inverse_M (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_DN_M_xeq_pM_inverse_M(int nc, void * r, void * a, void * b, int * index, int n);
/* replaces QLA_DN_M_xeq_pM_inverse_pM (lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135) */
void QLA_DN_M_xeq_pM_inverse_pM(int nc, void * r, void * a, void * b, int * index, int n);

#ifdef __cplusplus
}
#endif
#endif
