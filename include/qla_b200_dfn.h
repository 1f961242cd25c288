/*
 * qla_b200_dfn.h -- GENERATED by qla_b200/gen/gen_qla.py; do not edit.
 *
 * QLA DFN level-1 entry points implemented by libqla_b200.so (sm_100a).
 * Each declaration replaces the reference function of the same name, whose
 * C loop the reference generator emits from the cited section.  Array
 * arguments are device pointers; see qla_b200_runtime.h for scalars,
 * reduction outputs, streams and errors.
 */
#ifndef QLA_B200_DFN_H
#define QLA_B200_DFN_H
#include "qla_b200_types.h"

#ifdef __cplusplus
#define QLA_B200_RESTRICT __restrict__
extern "C" {
#else
#define QLA_B200_RESTRICT restrict
#endif

/* ---- norm2: replaces the DFN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DFN_r_veq_norm2_V (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DFN_r_veq_norm2_V(int nc, QLA_D_Real * r, void * a, int n);
/* replaces QLA_DFN_r_veq_norm2_pV (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DFN_r_veq_norm2_pV(int nc, QLA_D_Real * r, void * a, int n);
/* ---- dot: replaces the DFN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DFN_c_veq_V_dot_V (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_veq_V_dot_V(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DFN_c_veq_V_dot_pV (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_veq_V_dot_pV(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DFN_c_veq_pV_dot_V (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_veq_pV_dot_V(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DFN_c_veq_pV_dot_pV (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_veq_pV_dot_pV(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* ---- norm2: replaces the DFN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DFN_r_xeq_norm2_V (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DFN_r_xeq_norm2_V(int nc, QLA_D_Real * r, void * a, int * index, int n);
/* replaces QLA_DFN_r_xeq_norm2_pV (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DFN_r_xeq_norm2_pV(int nc, QLA_D_Real * r, void * a, int * index, int n);
/* ---- dot: replaces the DFN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DFN_c_xeq_V_dot_V (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_xeq_V_dot_V(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DFN_c_xeq_V_dot_pV (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_xeq_V_dot_pV(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DFN_c_xeq_pV_dot_V (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_xeq_pV_dot_V(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DFN_c_xeq_pV_dot_pV (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_xeq_pV_dot_pV(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* ---- norm2: replaces the DFN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DFN_r_veq_norm2_H (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DFN_r_veq_norm2_H(int nc, QLA_D_Real * r, void * a, int n);
/* replaces QLA_DFN_r_veq_norm2_pH (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DFN_r_veq_norm2_pH(int nc, QLA_D_Real * r, void * a, int n);
/* ---- dot: replaces the DFN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DFN_c_veq_H_dot_H (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_veq_H_dot_H(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DFN_c_veq_H_dot_pH (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_veq_H_dot_pH(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DFN_c_veq_pH_dot_H (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_veq_pH_dot_H(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DFN_c_veq_pH_dot_pH (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_veq_pH_dot_pH(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* ---- norm2: replaces the DFN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DFN_r_xeq_norm2_H (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DFN_r_xeq_norm2_H(int nc, QLA_D_Real * r, void * a, int * index, int n);
/* replaces QLA_DFN_r_xeq_norm2_pH (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DFN_r_xeq_norm2_pH(int nc, QLA_D_Real * r, void * a, int * index, int n);
/* ---- dot: replaces the DFN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DFN_c_xeq_H_dot_H (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_xeq_H_dot_H(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DFN_c_xeq_H_dot_pH (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_xeq_H_dot_pH(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DFN_c_xeq_pH_dot_H (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_xeq_pH_dot_H(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DFN_c_xeq_pH_dot_pH (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_xeq_pH_dot_pH(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* ---- norm2: replaces the DFN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DFN_r_veq_norm2_D (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DFN_r_veq_norm2_D(int nc, QLA_D_Real * r, void * a, int n);
/* replaces QLA_DFN_r_veq_norm2_pD (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DFN_r_veq_norm2_pD(int nc, QLA_D_Real * r, void * a, int n);
/* ---- dot: replaces the DFN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DFN_c_veq_D_dot_D (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_veq_D_dot_D(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DFN_c_veq_D_dot_pD (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_veq_D_dot_pD(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DFN_c_veq_pD_dot_D (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_veq_pD_dot_D(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DFN_c_veq_pD_dot_pD (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_veq_pD_dot_pD(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* ---- norm2: replaces the DFN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DFN_r_xeq_norm2_D (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DFN_r_xeq_norm2_D(int nc, QLA_D_Real * r, void * a, int * index, int n);
/* replaces QLA_DFN_r_xeq_norm2_pD (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DFN_r_xeq_norm2_pD(int nc, QLA_D_Real * r, void * a, int * index, int n);
/* ---- dot: replaces the DFN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DFN_c_xeq_D_dot_D (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_xeq_D_dot_D(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DFN_c_xeq_D_dot_pD (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_xeq_D_dot_pD(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DFN_c_xeq_pD_dot_D (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_xeq_pD_dot_D(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DFN_c_xeq_pD_dot_pD (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_xeq_pD_dot_pD(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* ---- norm2: replaces the DFN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DFN_r_veq_norm2_M (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DFN_r_veq_norm2_M(int nc, QLA_D_Real * r, void * a, int n);
/* replaces QLA_DFN_r_veq_norm2_pM (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DFN_r_veq_norm2_pM(int nc, QLA_D_Real * r, void * a, int n);
/* ---- dot: replaces the DFN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DFN_c_veq_M_dot_M (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_veq_M_dot_M(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DFN_c_veq_M_dot_pM (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_veq_M_dot_pM(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DFN_c_veq_pM_dot_M (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_veq_pM_dot_M(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* replaces QLA_DFN_c_veq_pM_dot_pM (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_veq_pM_dot_pM(int nc, QLA_D_Complex * r, void * a, void * b, int n);
/* ---- norm2: replaces the DFN functions emitted by lib/perl/build_qla.pl:2089-2155 */
/* replaces QLA_DFN_r_xeq_norm2_M (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DFN_r_xeq_norm2_M(int nc, QLA_D_Real * r, void * a, int * index, int n);
/* replaces QLA_DFN_r_xeq_norm2_pM (lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)) */
void QLA_DFN_r_xeq_norm2_pM(int nc, QLA_D_Real * r, void * a, int * index, int n);
/* ---- dot: replaces the DFN functions emitted by lib/perl/build_qla.pl:2196-2360 */
/* replaces QLA_DFN_c_xeq_M_dot_M (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_xeq_M_dot_M(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DFN_c_xeq_M_dot_pM (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_xeq_M_dot_pM(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DFN_c_xeq_pM_dot_M (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_xeq_pM_dot_M(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);
/* replaces QLA_DFN_c_xeq_pM_dot_pM (lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)) */
void QLA_DFN_c_xeq_pM_dot_pM(int nc, QLA_D_Complex * r, void * a, void * b, int * index, int n);

#ifdef __cplusplus
}
#endif
#endif
