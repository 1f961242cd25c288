// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F2 redot entry points (extern "C"), reference: lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"

extern "C" {
QLAB_EXPORT void QLA_F2_r_veq_re_V_dot_V(QLA_F_Real *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_r_veq_re_V_dot_V");
  qlab::api_reduce<qlab::ReDotOp<float, 2, float>>("F2_redot", r, sizeof(float), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_r_veq_re_V_dot_pV(QLA_F_Real *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_r_veq_re_V_dot_pV");
  qlab::api_reduce<qlab::ReDotOp<float, 2, float>>("F2_redot", r, sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_r_veq_re_pV_dot_V(QLA_F_Real *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_r_veq_re_pV_dot_V");
  qlab::api_reduce<qlab::ReDotOp<float, 2, float>>("F2_redot", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_r_veq_re_pV_dot_pV(QLA_F_Real *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_r_veq_re_pV_dot_pV");
  qlab::api_reduce<qlab::ReDotOp<float, 2, float>>("F2_redot", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_r_xeq_re_V_dot_V(QLA_F_Real *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_r_xeq_re_V_dot_V");
  qlab::api_reduce<qlab::ReDotOp<float, 2, float>>("F2_redot", r, sizeof(float), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_r_xeq_re_V_dot_pV(QLA_F_Real *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_r_xeq_re_V_dot_pV");
  qlab::api_reduce<qlab::ReDotOp<float, 2, float>>("F2_redot", r, sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_r_xeq_re_pV_dot_V(QLA_F_Real *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_r_xeq_re_pV_dot_V");
  qlab::api_reduce<qlab::ReDotOp<float, 2, float>>("F2_redot", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_r_xeq_re_pV_dot_pV(QLA_F_Real *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_r_xeq_re_pV_dot_pV");
  qlab::api_reduce<qlab::ReDotOp<float, 2, float>>("F2_redot", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_r_veq_re_V_dot_V(QLA_D_Real *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_r_veq_re_V_dot_V");
  qlab::api_reduce<qlab::ReDotOp<float, 2, double>>("F2_redot", r, sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_r_veq_re_V_dot_pV(QLA_D_Real *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_r_veq_re_V_dot_pV");
  qlab::api_reduce<qlab::ReDotOp<float, 2, double>>("F2_redot", r, sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_r_veq_re_pV_dot_V(QLA_D_Real *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_r_veq_re_pV_dot_V");
  qlab::api_reduce<qlab::ReDotOp<float, 2, double>>("F2_redot", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_r_veq_re_pV_dot_pV(QLA_D_Real *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_r_veq_re_pV_dot_pV");
  qlab::api_reduce<qlab::ReDotOp<float, 2, double>>("F2_redot", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_r_xeq_re_V_dot_V(QLA_D_Real *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_r_xeq_re_V_dot_V");
  qlab::api_reduce<qlab::ReDotOp<float, 2, double>>("F2_redot", r, sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_r_xeq_re_V_dot_pV(QLA_D_Real *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_r_xeq_re_V_dot_pV");
  qlab::api_reduce<qlab::ReDotOp<float, 2, double>>("F2_redot", r, sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_r_xeq_re_pV_dot_V(QLA_D_Real *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_r_xeq_re_pV_dot_V");
  qlab::api_reduce<qlab::ReDotOp<float, 2, double>>("F2_redot", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_r_xeq_re_pV_dot_pV(QLA_D_Real *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_r_xeq_re_pV_dot_pV");
  qlab::api_reduce<qlab::ReDotOp<float, 2, double>>("F2_redot", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_r_veq_re_H_dot_H(QLA_F_Real *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_r_veq_re_H_dot_H");
  qlab::api_reduce<qlab::ReDotOp<float, 4, float>>("F2_redot", r, sizeof(float), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_r_veq_re_H_dot_pH(QLA_F_Real *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_r_veq_re_H_dot_pH");
  qlab::api_reduce<qlab::ReDotOp<float, 4, float>>("F2_redot", r, sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_r_veq_re_pH_dot_H(QLA_F_Real *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_r_veq_re_pH_dot_H");
  qlab::api_reduce<qlab::ReDotOp<float, 4, float>>("F2_redot", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_r_veq_re_pH_dot_pH(QLA_F_Real *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_r_veq_re_pH_dot_pH");
  qlab::api_reduce<qlab::ReDotOp<float, 4, float>>("F2_redot", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_r_xeq_re_H_dot_H(QLA_F_Real *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_r_xeq_re_H_dot_H");
  qlab::api_reduce<qlab::ReDotOp<float, 4, float>>("F2_redot", r, sizeof(float), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_r_xeq_re_H_dot_pH(QLA_F_Real *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_r_xeq_re_H_dot_pH");
  qlab::api_reduce<qlab::ReDotOp<float, 4, float>>("F2_redot", r, sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_r_xeq_re_pH_dot_H(QLA_F_Real *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_r_xeq_re_pH_dot_H");
  qlab::api_reduce<qlab::ReDotOp<float, 4, float>>("F2_redot", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_r_xeq_re_pH_dot_pH(QLA_F_Real *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_r_xeq_re_pH_dot_pH");
  qlab::api_reduce<qlab::ReDotOp<float, 4, float>>("F2_redot", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_r_veq_re_H_dot_H(QLA_D_Real *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_r_veq_re_H_dot_H");
  qlab::api_reduce<qlab::ReDotOp<float, 4, double>>("F2_redot", r, sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_r_veq_re_H_dot_pH(QLA_D_Real *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_r_veq_re_H_dot_pH");
  qlab::api_reduce<qlab::ReDotOp<float, 4, double>>("F2_redot", r, sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_r_veq_re_pH_dot_H(QLA_D_Real *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_r_veq_re_pH_dot_H");
  qlab::api_reduce<qlab::ReDotOp<float, 4, double>>("F2_redot", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_r_veq_re_pH_dot_pH(QLA_D_Real *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_r_veq_re_pH_dot_pH");
  qlab::api_reduce<qlab::ReDotOp<float, 4, double>>("F2_redot", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_r_xeq_re_H_dot_H(QLA_D_Real *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_r_xeq_re_H_dot_H");
  qlab::api_reduce<qlab::ReDotOp<float, 4, double>>("F2_redot", r, sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_r_xeq_re_H_dot_pH(QLA_D_Real *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_r_xeq_re_H_dot_pH");
  qlab::api_reduce<qlab::ReDotOp<float, 4, double>>("F2_redot", r, sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_r_xeq_re_pH_dot_H(QLA_D_Real *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_r_xeq_re_pH_dot_H");
  qlab::api_reduce<qlab::ReDotOp<float, 4, double>>("F2_redot", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_r_xeq_re_pH_dot_pH(QLA_D_Real *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_r_xeq_re_pH_dot_pH");
  qlab::api_reduce<qlab::ReDotOp<float, 4, double>>("F2_redot", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_r_veq_re_D_dot_D(QLA_F_Real *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_r_veq_re_D_dot_D");
  qlab::api_reduce<qlab::ReDotOp<float, 8, float>>("F2_redot", r, sizeof(float), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_r_veq_re_D_dot_pD(QLA_F_Real *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_r_veq_re_D_dot_pD");
  qlab::api_reduce<qlab::ReDotOp<float, 8, float>>("F2_redot", r, sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_r_veq_re_pD_dot_D(QLA_F_Real *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_r_veq_re_pD_dot_D");
  qlab::api_reduce<qlab::ReDotOp<float, 8, float>>("F2_redot", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_r_veq_re_pD_dot_pD(QLA_F_Real *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_r_veq_re_pD_dot_pD");
  qlab::api_reduce<qlab::ReDotOp<float, 8, float>>("F2_redot", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_r_xeq_re_D_dot_D(QLA_F_Real *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_r_xeq_re_D_dot_D");
  qlab::api_reduce<qlab::ReDotOp<float, 8, float>>("F2_redot", r, sizeof(float), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_r_xeq_re_D_dot_pD(QLA_F_Real *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_r_xeq_re_D_dot_pD");
  qlab::api_reduce<qlab::ReDotOp<float, 8, float>>("F2_redot", r, sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_r_xeq_re_pD_dot_D(QLA_F_Real *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_r_xeq_re_pD_dot_D");
  qlab::api_reduce<qlab::ReDotOp<float, 8, float>>("F2_redot", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_r_xeq_re_pD_dot_pD(QLA_F_Real *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_r_xeq_re_pD_dot_pD");
  qlab::api_reduce<qlab::ReDotOp<float, 8, float>>("F2_redot", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_r_veq_re_D_dot_D(QLA_D_Real *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_r_veq_re_D_dot_D");
  qlab::api_reduce<qlab::ReDotOp<float, 8, double>>("F2_redot", r, sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_r_veq_re_D_dot_pD(QLA_D_Real *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_r_veq_re_D_dot_pD");
  qlab::api_reduce<qlab::ReDotOp<float, 8, double>>("F2_redot", r, sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_r_veq_re_pD_dot_D(QLA_D_Real *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_r_veq_re_pD_dot_D");
  qlab::api_reduce<qlab::ReDotOp<float, 8, double>>("F2_redot", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_r_veq_re_pD_dot_pD(QLA_D_Real *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_r_veq_re_pD_dot_pD");
  qlab::api_reduce<qlab::ReDotOp<float, 8, double>>("F2_redot", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_r_xeq_re_D_dot_D(QLA_D_Real *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_r_xeq_re_D_dot_D");
  qlab::api_reduce<qlab::ReDotOp<float, 8, double>>("F2_redot", r, sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_r_xeq_re_D_dot_pD(QLA_D_Real *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_r_xeq_re_D_dot_pD");
  qlab::api_reduce<qlab::ReDotOp<float, 8, double>>("F2_redot", r, sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_r_xeq_re_pD_dot_D(QLA_D_Real *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_r_xeq_re_pD_dot_D");
  qlab::api_reduce<qlab::ReDotOp<float, 8, double>>("F2_redot", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_r_xeq_re_pD_dot_pD(QLA_D_Real *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_r_xeq_re_pD_dot_pD");
  qlab::api_reduce<qlab::ReDotOp<float, 8, double>>("F2_redot", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_r_veq_re_M_dot_M(QLA_F_Real *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_r_veq_re_M_dot_M");
  qlab::api_reduce<qlab::ReDotOp<float, 4, float>>("F2_redot", r, sizeof(float), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_r_veq_re_M_dot_pM(QLA_F_Real *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_r_veq_re_M_dot_pM");
  qlab::api_reduce<qlab::ReDotOp<float, 4, float>>("F2_redot", r, sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_r_veq_re_pM_dot_M(QLA_F_Real *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_r_veq_re_pM_dot_M");
  qlab::api_reduce<qlab::ReDotOp<float, 4, float>>("F2_redot", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_r_veq_re_pM_dot_pM(QLA_F_Real *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_r_veq_re_pM_dot_pM");
  qlab::api_reduce<qlab::ReDotOp<float, 4, float>>("F2_redot", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_r_xeq_re_M_dot_M(QLA_F_Real *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_r_xeq_re_M_dot_M");
  qlab::api_reduce<qlab::ReDotOp<float, 4, float>>("F2_redot", r, sizeof(float), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_r_xeq_re_M_dot_pM(QLA_F_Real *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_r_xeq_re_M_dot_pM");
  qlab::api_reduce<qlab::ReDotOp<float, 4, float>>("F2_redot", r, sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_r_xeq_re_pM_dot_M(QLA_F_Real *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_r_xeq_re_pM_dot_M");
  qlab::api_reduce<qlab::ReDotOp<float, 4, float>>("F2_redot", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_r_xeq_re_pM_dot_pM(QLA_F_Real *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_r_xeq_re_pM_dot_pM");
  qlab::api_reduce<qlab::ReDotOp<float, 4, float>>("F2_redot", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_r_veq_re_M_dot_M(QLA_D_Real *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_r_veq_re_M_dot_M");
  qlab::api_reduce<qlab::ReDotOp<float, 4, double>>("F2_redot", r, sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_r_veq_re_M_dot_pM(QLA_D_Real *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_r_veq_re_M_dot_pM");
  qlab::api_reduce<qlab::ReDotOp<float, 4, double>>("F2_redot", r, sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_r_veq_re_pM_dot_M(QLA_D_Real *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_r_veq_re_pM_dot_M");
  qlab::api_reduce<qlab::ReDotOp<float, 4, double>>("F2_redot", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_r_veq_re_pM_dot_pM(QLA_D_Real *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_r_veq_re_pM_dot_pM");
  qlab::api_reduce<qlab::ReDotOp<float, 4, double>>("F2_redot", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_r_xeq_re_M_dot_M(QLA_D_Real *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_r_xeq_re_M_dot_M");
  qlab::api_reduce<qlab::ReDotOp<float, 4, double>>("F2_redot", r, sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_r_xeq_re_M_dot_pM(QLA_D_Real *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_r_xeq_re_M_dot_pM");
  qlab::api_reduce<qlab::ReDotOp<float, 4, double>>("F2_redot", r, sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_r_xeq_re_pM_dot_M(QLA_D_Real *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_r_xeq_re_pM_dot_M");
  qlab::api_reduce<qlab::ReDotOp<float, 4, double>>("F2_redot", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_r_xeq_re_pM_dot_pM(QLA_D_Real *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_r_xeq_re_pM_dot_pM");
  qlab::api_reduce<qlab::ReDotOp<float, 4, double>>("F2_redot", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

}  // extern "C"
