/*
 * qla_b200_df2.h -- GENERATED by qla_b200/gen/gen_qla.py; do not edit.
 *
 * QLA DF2 level-1 entry points implemented by libqla_b200.so (sm_100a).
 * Each declaration replaces the reference function of the same name, whose
 * C loop the reference generator emits from the cited section.  Array
 * arguments are device pointers; see qla_b200_runtime.h for scalars,
 * reduction outputs, streams and errors.
 */
#ifndef QLA_B200_DF2_H
#define QLA_B200_DF2_H
#include "qla_b200_types.h"

#ifdef __cplusplus
#define QLA_B200_RESTRICT __restrict__
extern "C" {
#else
#define QLA_B200_RESTRICT restrict
#endif

/* ---- norm2: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DF2_r_veq_norm2_V (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DF2_r_veq_norm2_V(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT a, int n);
/* replaces QLA_DF2_r_veq_norm2_pV (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DF2_r_veq_norm2_pV(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT * a, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_veq_V_dot_V (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_veq_V_dot_V(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT a, QLA_F2_ColorVector *QLA_B200_RESTRICT b, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_veq_re_V_dot_V (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_veq_re_V_dot_V(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT a, QLA_F2_ColorVector *QLA_B200_RESTRICT b, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_veq_V_dot_pV (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_veq_V_dot_pV(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT a, QLA_F2_ColorVector *QLA_B200_RESTRICT * b, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_veq_re_V_dot_pV (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_veq_re_V_dot_pV(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT a, QLA_F2_ColorVector *QLA_B200_RESTRICT * b, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_veq_pV_dot_V (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_veq_pV_dot_V(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT * a, QLA_F2_ColorVector *QLA_B200_RESTRICT b, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_veq_re_pV_dot_V (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_veq_re_pV_dot_V(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT * a, QLA_F2_ColorVector *QLA_B200_RESTRICT b, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_veq_pV_dot_pV (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_veq_pV_dot_pV(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT * a, QLA_F2_ColorVector *QLA_B200_RESTRICT * b, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_veq_re_pV_dot_pV (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_veq_re_pV_dot_pV(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT * a, QLA_F2_ColorVector *QLA_B200_RESTRICT * b, int n);
/* ---- norm2: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DF2_r_xeq_norm2_V (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DF2_r_xeq_norm2_V(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_DF2_r_xeq_norm2_pV (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DF2_r_xeq_norm2_pV(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT * a, int * index, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_xeq_V_dot_V (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_xeq_V_dot_V(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT a, QLA_F2_ColorVector *QLA_B200_RESTRICT b, int * index, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_xeq_re_V_dot_V (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_xeq_re_V_dot_V(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT a, QLA_F2_ColorVector *QLA_B200_RESTRICT b, int * index, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_xeq_V_dot_pV (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_xeq_V_dot_pV(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT a, QLA_F2_ColorVector *QLA_B200_RESTRICT * b, int * index, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_xeq_re_V_dot_pV (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_xeq_re_V_dot_pV(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT a, QLA_F2_ColorVector *QLA_B200_RESTRICT * b, int * index, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_xeq_pV_dot_V (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_xeq_pV_dot_V(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT * a, QLA_F2_ColorVector *QLA_B200_RESTRICT b, int * index, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_xeq_re_pV_dot_V (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_xeq_re_pV_dot_V(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT * a, QLA_F2_ColorVector *QLA_B200_RESTRICT b, int * index, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_xeq_pV_dot_pV (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_xeq_pV_dot_pV(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT * a, QLA_F2_ColorVector *QLA_B200_RESTRICT * b, int * index, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_xeq_re_pV_dot_pV (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_xeq_re_pV_dot_pV(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT * a, QLA_F2_ColorVector *QLA_B200_RESTRICT * b, int * index, int n);
/* ---- norm2: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DF2_r_veq_norm2_H (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DF2_r_veq_norm2_H(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT a, int n);
/* replaces QLA_DF2_r_veq_norm2_pH (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DF2_r_veq_norm2_pH(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT * a, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_veq_H_dot_H (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_veq_H_dot_H(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT a, QLA_F2_HalfFermion *QLA_B200_RESTRICT b, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_veq_re_H_dot_H (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_veq_re_H_dot_H(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT a, QLA_F2_HalfFermion *QLA_B200_RESTRICT b, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_veq_H_dot_pH (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_veq_H_dot_pH(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT a, QLA_F2_HalfFermion *QLA_B200_RESTRICT * b, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_veq_re_H_dot_pH (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_veq_re_H_dot_pH(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT a, QLA_F2_HalfFermion *QLA_B200_RESTRICT * b, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_veq_pH_dot_H (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_veq_pH_dot_H(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT * a, QLA_F2_HalfFermion *QLA_B200_RESTRICT b, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_veq_re_pH_dot_H (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_veq_re_pH_dot_H(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT * a, QLA_F2_HalfFermion *QLA_B200_RESTRICT b, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_veq_pH_dot_pH (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_veq_pH_dot_pH(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT * a, QLA_F2_HalfFermion *QLA_B200_RESTRICT * b, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_veq_re_pH_dot_pH (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_veq_re_pH_dot_pH(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT * a, QLA_F2_HalfFermion *QLA_B200_RESTRICT * b, int n);
/* ---- norm2: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DF2_r_xeq_norm2_H (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DF2_r_xeq_norm2_H(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_DF2_r_xeq_norm2_pH (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DF2_r_xeq_norm2_pH(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT * a, int * index, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_xeq_H_dot_H (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_xeq_H_dot_H(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT a, QLA_F2_HalfFermion *QLA_B200_RESTRICT b, int * index, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_xeq_re_H_dot_H (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_xeq_re_H_dot_H(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT a, QLA_F2_HalfFermion *QLA_B200_RESTRICT b, int * index, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_xeq_H_dot_pH (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_xeq_H_dot_pH(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT a, QLA_F2_HalfFermion *QLA_B200_RESTRICT * b, int * index, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_xeq_re_H_dot_pH (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_xeq_re_H_dot_pH(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT a, QLA_F2_HalfFermion *QLA_B200_RESTRICT * b, int * index, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_xeq_pH_dot_H (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_xeq_pH_dot_H(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT * a, QLA_F2_HalfFermion *QLA_B200_RESTRICT b, int * index, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_xeq_re_pH_dot_H (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_xeq_re_pH_dot_H(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT * a, QLA_F2_HalfFermion *QLA_B200_RESTRICT b, int * index, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_xeq_pH_dot_pH (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_xeq_pH_dot_pH(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT * a, QLA_F2_HalfFermion *QLA_B200_RESTRICT * b, int * index, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_xeq_re_pH_dot_pH (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_xeq_re_pH_dot_pH(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT * a, QLA_F2_HalfFermion *QLA_B200_RESTRICT * b, int * index, int n);
/* ---- norm2: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DF2_r_veq_norm2_D (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DF2_r_veq_norm2_D(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT a, int n);
/* replaces QLA_DF2_r_veq_norm2_pD (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DF2_r_veq_norm2_pD(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT * a, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_veq_D_dot_D (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_veq_D_dot_D(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT a, QLA_F2_DiracFermion *QLA_B200_RESTRICT b, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_veq_re_D_dot_D (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_veq_re_D_dot_D(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT a, QLA_F2_DiracFermion *QLA_B200_RESTRICT b, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_veq_D_dot_pD (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_veq_D_dot_pD(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT a, QLA_F2_DiracFermion *QLA_B200_RESTRICT * b, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_veq_re_D_dot_pD (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_veq_re_D_dot_pD(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT a, QLA_F2_DiracFermion *QLA_B200_RESTRICT * b, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_veq_pD_dot_D (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_veq_pD_dot_D(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT * a, QLA_F2_DiracFermion *QLA_B200_RESTRICT b, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_veq_re_pD_dot_D (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_veq_re_pD_dot_D(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT * a, QLA_F2_DiracFermion *QLA_B200_RESTRICT b, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_veq_pD_dot_pD (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_veq_pD_dot_pD(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT * a, QLA_F2_DiracFermion *QLA_B200_RESTRICT * b, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_veq_re_pD_dot_pD (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_veq_re_pD_dot_pD(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT * a, QLA_F2_DiracFermion *QLA_B200_RESTRICT * b, int n);
/* ---- norm2: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DF2_r_xeq_norm2_D (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DF2_r_xeq_norm2_D(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_DF2_r_xeq_norm2_pD (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DF2_r_xeq_norm2_pD(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT * a, int * index, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_xeq_D_dot_D (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_xeq_D_dot_D(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT a, QLA_F2_DiracFermion *QLA_B200_RESTRICT b, int * index, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_xeq_re_D_dot_D (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_xeq_re_D_dot_D(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT a, QLA_F2_DiracFermion *QLA_B200_RESTRICT b, int * index, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_xeq_D_dot_pD (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_xeq_D_dot_pD(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT a, QLA_F2_DiracFermion *QLA_B200_RESTRICT * b, int * index, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_xeq_re_D_dot_pD (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_xeq_re_D_dot_pD(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT a, QLA_F2_DiracFermion *QLA_B200_RESTRICT * b, int * index, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_xeq_pD_dot_D (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_xeq_pD_dot_D(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT * a, QLA_F2_DiracFermion *QLA_B200_RESTRICT b, int * index, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_xeq_re_pD_dot_D (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_xeq_re_pD_dot_D(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT * a, QLA_F2_DiracFermion *QLA_B200_RESTRICT b, int * index, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_xeq_pD_dot_pD (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_xeq_pD_dot_pD(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT * a, QLA_F2_DiracFermion *QLA_B200_RESTRICT * b, int * index, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_xeq_re_pD_dot_pD (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_xeq_re_pD_dot_pD(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT * a, QLA_F2_DiracFermion *QLA_B200_RESTRICT * b, int * index, int n);
/* ---- norm2: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DF2_r_veq_norm2_M (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DF2_r_veq_norm2_M(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT a, int n);
/* replaces QLA_DF2_r_veq_norm2_pM (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DF2_r_veq_norm2_pM(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * a, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_veq_M_dot_M (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_veq_M_dot_M(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT b, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_veq_re_M_dot_M (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_veq_re_M_dot_M(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT b, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_veq_M_dot_pM (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_veq_M_dot_pM(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * b, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_veq_re_M_dot_pM (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_veq_re_M_dot_pM(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * b, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_veq_pM_dot_M (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_veq_pM_dot_M(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT b, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_veq_re_pM_dot_M (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_veq_re_pM_dot_M(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT b, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_veq_pM_dot_pM (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_veq_pM_dot_pM(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * b, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_veq_re_pM_dot_pM (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_veq_re_pM_dot_pM(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * b, int n);
/* ---- norm2: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DF2_r_xeq_norm2_M (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DF2_r_xeq_norm2_M(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_DF2_r_xeq_norm2_pM (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DF2_r_xeq_norm2_pM(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * a, int * index, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_xeq_M_dot_M (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_xeq_M_dot_M(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT b, int * index, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_xeq_re_M_dot_M (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_xeq_re_M_dot_M(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT b, int * index, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_xeq_M_dot_pM (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_xeq_M_dot_pM(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * b, int * index, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_xeq_re_M_dot_pM (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_xeq_re_M_dot_pM(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * b, int * index, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_xeq_pM_dot_M (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_xeq_pM_dot_M(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT b, int * index, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_xeq_re_pM_dot_M (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_xeq_re_pM_dot_M(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT b, int * index, int n);
/* ---- dot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DF2_c_xeq_pM_dot_pM (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DF2_c_xeq_pM_dot_pM(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * b, int * index, int n);
/* ---- redot: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2250-2284 (real part of the global inner product) */
/* replaces QLA_DF2_r_xeq_re_pM_dot_pM (lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)) */
void QLA_DF2_r_xeq_re_pM_dot_pM(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * b, int * index, int n);
/* ---- gred: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators */
/* replaces QLA_DF2_c_veq_Ma_dot_M (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_veq_Ma_dot_M(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT b, int n);
/* replaces QLA_DF2_c_veq_Ma_dot_pM (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_veq_Ma_dot_pM(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_DF2_c_veq_pMa_dot_M (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_veq_pMa_dot_M(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT b, int n);
/* replaces QLA_DF2_c_veq_pMa_dot_pM (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_veq_pMa_dot_pM(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_DF2_c_veq_P_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_veq_P_dot_P(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT b, int n);
/* replaces QLA_DF2_c_veq_P_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_veq_P_dot_pP(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_DF2_c_veq_pP_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_veq_pP_dot_P(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT b, int n);
/* replaces QLA_DF2_c_veq_pP_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_veq_pP_dot_pP(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_DF2_c_veq_Pa_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_veq_Pa_dot_P(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT b, int n);
/* replaces QLA_DF2_c_veq_Pa_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_veq_Pa_dot_pP(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_DF2_c_veq_pPa_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_veq_pPa_dot_P(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT b, int n);
/* replaces QLA_DF2_c_veq_pPa_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_veq_pPa_dot_pP(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_DF2_r_veq_re_P_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_r_veq_re_P_dot_P(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT b, int n);
/* replaces QLA_DF2_r_veq_re_P_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_r_veq_re_P_dot_pP(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_DF2_r_veq_re_pP_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_r_veq_re_pP_dot_P(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT b, int n);
/* replaces QLA_DF2_r_veq_re_pP_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_r_veq_re_pP_dot_pP(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * b, int n);
/* replaces QLA_DF2_r_veq_norm2_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_r_veq_norm2_P(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT a, int n);
/* replaces QLA_DF2_r_veq_norm2_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_r_veq_norm2_pP(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * a, int n);
/* ---- gsum: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites) */
/* replaces QLA_DF2_v_veq_sum_V (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_DF2_v_veq_sum_V(QLA_D2_ColorVector *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT a, int n);
/* replaces QLA_DF2_v_veq_sum_pV (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_DF2_v_veq_sum_pV(QLA_D2_ColorVector *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_DF2_h_veq_sum_H (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_DF2_h_veq_sum_H(QLA_D2_HalfFermion *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT a, int n);
/* replaces QLA_DF2_h_veq_sum_pH (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_DF2_h_veq_sum_pH(QLA_D2_HalfFermion *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_DF2_d_veq_sum_D (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_DF2_d_veq_sum_D(QLA_D2_DiracFermion *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT a, int n);
/* replaces QLA_DF2_d_veq_sum_pD (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_DF2_d_veq_sum_pD(QLA_D2_DiracFermion *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_DF2_m_veq_sum_M (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_DF2_m_veq_sum_M(QLA_D2_ColorMatrix *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT a, int n);
/* replaces QLA_DF2_m_veq_sum_pM (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_DF2_m_veq_sum_pM(QLA_D2_ColorMatrix *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_DF2_p_veq_sum_P (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_DF2_p_veq_sum_P(QLA_D2_DiracPropagator *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT a, int n);
/* replaces QLA_DF2_p_veq_sum_pP (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_DF2_p_veq_sum_pP(QLA_D2_DiracPropagator *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * a, int n);
/* ---- convert: replaces the DF2 functions emitted by lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion */
/* replaces QLA_DF2_V_veq_V (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_DF2_V_veq_V(QLA_D2_ColorVector *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT a, int n);
/* replaces QLA_FD2_V_veq_V (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_FD2_V_veq_V(QLA_F2_ColorVector *QLA_B200_RESTRICT r, QLA_D2_ColorVector *QLA_B200_RESTRICT a, int n);
/* replaces QLA_DF2_V_veq_pV (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_DF2_V_veq_pV(QLA_D2_ColorVector *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_FD2_V_veq_pV (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_FD2_V_veq_pV(QLA_F2_ColorVector *QLA_B200_RESTRICT r, QLA_D2_ColorVector *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_DF2_H_veq_H (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_DF2_H_veq_H(QLA_D2_HalfFermion *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT a, int n);
/* replaces QLA_FD2_H_veq_H (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_FD2_H_veq_H(QLA_F2_HalfFermion *QLA_B200_RESTRICT r, QLA_D2_HalfFermion *QLA_B200_RESTRICT a, int n);
/* replaces QLA_DF2_H_veq_pH (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_DF2_H_veq_pH(QLA_D2_HalfFermion *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_FD2_H_veq_pH (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_FD2_H_veq_pH(QLA_F2_HalfFermion *QLA_B200_RESTRICT r, QLA_D2_HalfFermion *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_DF2_D_veq_D (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_DF2_D_veq_D(QLA_D2_DiracFermion *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT a, int n);
/* replaces QLA_FD2_D_veq_D (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_FD2_D_veq_D(QLA_F2_DiracFermion *QLA_B200_RESTRICT r, QLA_D2_DiracFermion *QLA_B200_RESTRICT a, int n);
/* replaces QLA_DF2_D_veq_pD (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_DF2_D_veq_pD(QLA_D2_DiracFermion *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_FD2_D_veq_pD (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_FD2_D_veq_pD(QLA_F2_DiracFermion *QLA_B200_RESTRICT r, QLA_D2_DiracFermion *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_DF2_M_veq_M (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_DF2_M_veq_M(QLA_D2_ColorMatrix *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT a, int n);
/* replaces QLA_FD2_M_veq_M (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_FD2_M_veq_M(QLA_F2_ColorMatrix *QLA_B200_RESTRICT r, QLA_D2_ColorMatrix *QLA_B200_RESTRICT a, int n);
/* replaces QLA_DF2_M_veq_pM (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_DF2_M_veq_pM(QLA_D2_ColorMatrix *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_FD2_M_veq_pM (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_FD2_M_veq_pM(QLA_F2_ColorMatrix *QLA_B200_RESTRICT r, QLA_D2_ColorMatrix *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_DF2_P_veq_P (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_DF2_P_veq_P(QLA_D2_DiracPropagator *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT a, int n);
/* replaces QLA_FD2_P_veq_P (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_FD2_P_veq_P(QLA_F2_DiracPropagator *QLA_B200_RESTRICT r, QLA_D2_DiracPropagator *QLA_B200_RESTRICT a, int n);
/* replaces QLA_DF2_P_veq_pP (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_DF2_P_veq_pP(QLA_D2_DiracPropagator *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * a, int n);
/* replaces QLA_FD2_P_veq_pP (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_FD2_P_veq_pP(QLA_F2_DiracPropagator *QLA_B200_RESTRICT r, QLA_D2_DiracPropagator *QLA_B200_RESTRICT * a, int n);
/* ---- gred: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators */
/* replaces QLA_DF2_c_xeq_Ma_dot_M (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_xeq_Ma_dot_M(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_DF2_c_xeq_Ma_dot_pM (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_xeq_Ma_dot_pM(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_DF2_c_xeq_pMa_dot_M (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_xeq_pMa_dot_M(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_DF2_c_xeq_pMa_dot_pM (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_xeq_pMa_dot_pM(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * a, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_DF2_c_xeq_P_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_xeq_P_dot_P(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_DF2_c_xeq_P_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_xeq_P_dot_pP(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_DF2_c_xeq_pP_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_xeq_pP_dot_P(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_DF2_c_xeq_pP_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_xeq_pP_dot_pP(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_DF2_c_xeq_Pa_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_xeq_Pa_dot_P(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_DF2_c_xeq_Pa_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_xeq_Pa_dot_pP(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_DF2_c_xeq_pPa_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_xeq_pPa_dot_P(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_DF2_c_xeq_pPa_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_c_xeq_pPa_dot_pP(QLA_D_Complex *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_DF2_r_xeq_re_P_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_r_xeq_re_P_dot_P(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_DF2_r_xeq_re_P_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_r_xeq_re_P_dot_pP(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_DF2_r_xeq_re_pP_dot_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_r_xeq_re_pP_dot_P(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT b, int * index, int n);
/* replaces QLA_DF2_r_xeq_re_pP_dot_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_r_xeq_re_pP_dot_pP(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * a, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * b, int * index, int n);
/* replaces QLA_DF2_r_xeq_norm2_P (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_r_xeq_norm2_P(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_DF2_r_xeq_norm2_pP (lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, trace of the adjoint-form products Ma.M and Pa.P)) */
void QLA_DF2_r_xeq_norm2_pP(QLA_D_Real *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * a, int * index, int n);
/* ---- gsum: replaces the DF2 functions emitted by lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites) */
/* replaces QLA_DF2_v_xeq_sum_V (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_DF2_v_xeq_sum_V(QLA_D2_ColorVector *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_DF2_v_xeq_sum_pV (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_DF2_v_xeq_sum_pV(QLA_D2_ColorVector *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_DF2_h_xeq_sum_H (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_DF2_h_xeq_sum_H(QLA_D2_HalfFermion *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_DF2_h_xeq_sum_pH (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_DF2_h_xeq_sum_pH(QLA_D2_HalfFermion *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_DF2_d_xeq_sum_D (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_DF2_d_xeq_sum_D(QLA_D2_DiracFermion *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_DF2_d_xeq_sum_pD (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_DF2_d_xeq_sum_pD(QLA_D2_DiracFermion *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_DF2_m_xeq_sum_M (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_DF2_m_xeq_sum_M(QLA_D2_ColorMatrix *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_DF2_m_xeq_sum_pM (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_DF2_m_xeq_sum_pM(QLA_D2_ColorMatrix *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_DF2_p_xeq_sum_P (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_DF2_p_xeq_sum_P(QLA_D2_DiracPropagator *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_DF2_p_xeq_sum_pP (lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)) */
void QLA_DF2_p_xeq_sum_pP(QLA_D2_DiracPropagator *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * a, int * index, int n);
/* ---- convert: replaces the DF2 functions emitted by lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion */
/* replaces QLA_DF2_V_xeq_V (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_DF2_V_xeq_V(QLA_D2_ColorVector *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_FD2_V_xeq_V (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_FD2_V_xeq_V(QLA_F2_ColorVector *QLA_B200_RESTRICT r, QLA_D2_ColorVector *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_DF2_V_xeq_pV (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_DF2_V_xeq_pV(QLA_D2_ColorVector *QLA_B200_RESTRICT r, QLA_F2_ColorVector *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_FD2_V_xeq_pV (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_FD2_V_xeq_pV(QLA_F2_ColorVector *QLA_B200_RESTRICT r, QLA_D2_ColorVector *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_DF2_H_xeq_H (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_DF2_H_xeq_H(QLA_D2_HalfFermion *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_FD2_H_xeq_H (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_FD2_H_xeq_H(QLA_F2_HalfFermion *QLA_B200_RESTRICT r, QLA_D2_HalfFermion *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_DF2_H_xeq_pH (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_DF2_H_xeq_pH(QLA_D2_HalfFermion *QLA_B200_RESTRICT r, QLA_F2_HalfFermion *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_FD2_H_xeq_pH (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_FD2_H_xeq_pH(QLA_F2_HalfFermion *QLA_B200_RESTRICT r, QLA_D2_HalfFermion *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_DF2_D_xeq_D (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_DF2_D_xeq_D(QLA_D2_DiracFermion *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_FD2_D_xeq_D (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_FD2_D_xeq_D(QLA_F2_DiracFermion *QLA_B200_RESTRICT r, QLA_D2_DiracFermion *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_DF2_D_xeq_pD (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_DF2_D_xeq_pD(QLA_D2_DiracFermion *QLA_B200_RESTRICT r, QLA_F2_DiracFermion *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_FD2_D_xeq_pD (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_FD2_D_xeq_pD(QLA_F2_DiracFermion *QLA_B200_RESTRICT r, QLA_D2_DiracFermion *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_DF2_M_xeq_M (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_DF2_M_xeq_M(QLA_D2_ColorMatrix *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_FD2_M_xeq_M (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_FD2_M_xeq_M(QLA_F2_ColorMatrix *QLA_B200_RESTRICT r, QLA_D2_ColorMatrix *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_DF2_M_xeq_pM (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_DF2_M_xeq_pM(QLA_D2_ColorMatrix *QLA_B200_RESTRICT r, QLA_F2_ColorMatrix *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_FD2_M_xeq_pM (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_FD2_M_xeq_pM(QLA_F2_ColorMatrix *QLA_B200_RESTRICT r, QLA_D2_ColorMatrix *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_DF2_P_xeq_P (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_DF2_P_xeq_P(QLA_D2_DiracPropagator *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_FD2_P_xeq_P (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_FD2_P_xeq_P(QLA_F2_DiracPropagator *QLA_B200_RESTRICT r, QLA_D2_DiracPropagator *QLA_B200_RESTRICT a, int * index, int n);
/* replaces QLA_DF2_P_xeq_pP (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_DF2_P_xeq_pP(QLA_D2_DiracPropagator *QLA_B200_RESTRICT r, QLA_F2_DiracPropagator *QLA_B200_RESTRICT * a, int * index, int n);
/* replaces QLA_FD2_P_xeq_pP (lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)) */
void QLA_FD2_P_xeq_pP(QLA_F2_DiracPropagator *QLA_B200_RESTRICT r, QLA_D2_DiracPropagator *QLA_B200_RESTRICT * a, int * index, int n);

#ifdef __cplusplus
}
#endif
#endif
