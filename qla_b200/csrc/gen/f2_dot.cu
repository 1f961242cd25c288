// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F2 dot entry points (extern "C"), reference: lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"

extern "C" {
QLAB_EXPORT void QLA_F2_c_veq_V_dot_V(QLA_F_Complex *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_V_dot_V");
  qlab::api_reduce<qlab::DotOp<float, 2, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_veq_V_dot_pV(QLA_F_Complex *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_V_dot_pV");
  qlab::api_reduce<qlab::DotOp<float, 2, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_veq_pV_dot_V(QLA_F_Complex *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_pV_dot_V");
  qlab::api_reduce<qlab::DotOp<float, 2, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_veq_pV_dot_pV(QLA_F_Complex *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_pV_dot_pV");
  qlab::api_reduce<qlab::DotOp<float, 2, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_V_dot_V(QLA_F_Complex *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_V_dot_V");
  qlab::api_reduce<qlab::DotOp<float, 2, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_V_dot_pV(QLA_F_Complex *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_V_dot_pV");
  qlab::api_reduce<qlab::DotOp<float, 2, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_pV_dot_V(QLA_F_Complex *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_pV_dot_V");
  qlab::api_reduce<qlab::DotOp<float, 2, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_pV_dot_pV(QLA_F_Complex *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_pV_dot_pV");
  qlab::api_reduce<qlab::DotOp<float, 2, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_V_dot_V(QLA_D_Complex *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_V_dot_V");
  qlab::api_reduce<qlab::DotOp<float, 2, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_V_dot_pV(QLA_D_Complex *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_V_dot_pV");
  qlab::api_reduce<qlab::DotOp<float, 2, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_pV_dot_V(QLA_D_Complex *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_pV_dot_V");
  qlab::api_reduce<qlab::DotOp<float, 2, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_pV_dot_pV(QLA_D_Complex *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_pV_dot_pV");
  qlab::api_reduce<qlab::DotOp<float, 2, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_V_dot_V(QLA_D_Complex *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_V_dot_V");
  qlab::api_reduce<qlab::DotOp<float, 2, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_V_dot_pV(QLA_D_Complex *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_V_dot_pV");
  qlab::api_reduce<qlab::DotOp<float, 2, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_pV_dot_V(QLA_D_Complex *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_pV_dot_V");
  qlab::api_reduce<qlab::DotOp<float, 2, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_pV_dot_pV(QLA_D_Complex *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, QLA_F2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_pV_dot_pV");
  qlab::api_reduce<qlab::DotOp<float, 2, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_c_veq_H_dot_H(QLA_F_Complex *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_H_dot_H");
  qlab::api_reduce<qlab::DotOp<float, 4, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_veq_H_dot_pH(QLA_F_Complex *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_H_dot_pH");
  qlab::api_reduce<qlab::DotOp<float, 4, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_veq_pH_dot_H(QLA_F_Complex *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_pH_dot_H");
  qlab::api_reduce<qlab::DotOp<float, 4, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_veq_pH_dot_pH(QLA_F_Complex *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_pH_dot_pH");
  qlab::api_reduce<qlab::DotOp<float, 4, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_H_dot_H(QLA_F_Complex *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_H_dot_H");
  qlab::api_reduce<qlab::DotOp<float, 4, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_H_dot_pH(QLA_F_Complex *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_H_dot_pH");
  qlab::api_reduce<qlab::DotOp<float, 4, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_pH_dot_H(QLA_F_Complex *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_pH_dot_H");
  qlab::api_reduce<qlab::DotOp<float, 4, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_pH_dot_pH(QLA_F_Complex *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_pH_dot_pH");
  qlab::api_reduce<qlab::DotOp<float, 4, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_H_dot_H(QLA_D_Complex *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_H_dot_H");
  qlab::api_reduce<qlab::DotOp<float, 4, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_H_dot_pH(QLA_D_Complex *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_H_dot_pH");
  qlab::api_reduce<qlab::DotOp<float, 4, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_pH_dot_H(QLA_D_Complex *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_pH_dot_H");
  qlab::api_reduce<qlab::DotOp<float, 4, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_pH_dot_pH(QLA_D_Complex *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_pH_dot_pH");
  qlab::api_reduce<qlab::DotOp<float, 4, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_H_dot_H(QLA_D_Complex *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, QLA_F2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_H_dot_H");
  qlab::api_reduce<qlab::DotOp<float, 4, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_H_dot_pH(QLA_D_Complex *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, QLA_F2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_H_dot_pH");
  qlab::api_reduce<qlab::DotOp<float, 4, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_pH_dot_H(QLA_D_Complex *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_pH_dot_H");
  qlab::api_reduce<qlab::DotOp<float, 4, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_pH_dot_pH(QLA_D_Complex *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, QLA_F2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_pH_dot_pH");
  qlab::api_reduce<qlab::DotOp<float, 4, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_c_veq_D_dot_D(QLA_F_Complex *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_D_dot_D");
  qlab::api_reduce<qlab::DotOp<float, 8, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_veq_D_dot_pD(QLA_F_Complex *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_D_dot_pD");
  qlab::api_reduce<qlab::DotOp<float, 8, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_veq_pD_dot_D(QLA_F_Complex *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_pD_dot_D");
  qlab::api_reduce<qlab::DotOp<float, 8, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_veq_pD_dot_pD(QLA_F_Complex *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_pD_dot_pD");
  qlab::api_reduce<qlab::DotOp<float, 8, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_D_dot_D(QLA_F_Complex *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_D_dot_D");
  qlab::api_reduce<qlab::DotOp<float, 8, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_D_dot_pD(QLA_F_Complex *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_D_dot_pD");
  qlab::api_reduce<qlab::DotOp<float, 8, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_pD_dot_D(QLA_F_Complex *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_pD_dot_D");
  qlab::api_reduce<qlab::DotOp<float, 8, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_pD_dot_pD(QLA_F_Complex *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_pD_dot_pD");
  qlab::api_reduce<qlab::DotOp<float, 8, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_D_dot_D(QLA_D_Complex *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_D_dot_D");
  qlab::api_reduce<qlab::DotOp<float, 8, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_D_dot_pD(QLA_D_Complex *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_D_dot_pD");
  qlab::api_reduce<qlab::DotOp<float, 8, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_pD_dot_D(QLA_D_Complex *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_pD_dot_D");
  qlab::api_reduce<qlab::DotOp<float, 8, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_pD_dot_pD(QLA_D_Complex *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_pD_dot_pD");
  qlab::api_reduce<qlab::DotOp<float, 8, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_D_dot_D(QLA_D_Complex *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, QLA_F2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_D_dot_D");
  qlab::api_reduce<qlab::DotOp<float, 8, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_D_dot_pD(QLA_D_Complex *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, QLA_F2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_D_dot_pD");
  qlab::api_reduce<qlab::DotOp<float, 8, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_pD_dot_D(QLA_D_Complex *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_pD_dot_D");
  qlab::api_reduce<qlab::DotOp<float, 8, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_pD_dot_pD(QLA_D_Complex *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, QLA_F2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_pD_dot_pD");
  qlab::api_reduce<qlab::DotOp<float, 8, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_c_veq_M_dot_M(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_M_dot_M");
  qlab::api_reduce<qlab::DotOp<float, 4, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_veq_M_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_M_dot_pM");
  qlab::api_reduce<qlab::DotOp<float, 4, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_veq_pM_dot_M(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_pM_dot_M");
  qlab::api_reduce<qlab::DotOp<float, 4, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_veq_pM_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F2_c_veq_pM_dot_pM");
  qlab::api_reduce<qlab::DotOp<float, 4, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_M_dot_M(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_M_dot_M");
  qlab::api_reduce<qlab::DotOp<float, 4, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_M_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_M_dot_pM");
  qlab::api_reduce<qlab::DotOp<float, 4, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_pM_dot_M(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_pM_dot_M");
  qlab::api_reduce<qlab::DotOp<float, 4, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F2_c_xeq_pM_dot_pM(QLA_F_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F2_c_xeq_pM_dot_pM");
  qlab::api_reduce<qlab::DotOp<float, 4, float>>("F2_dot", r, 2 * sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_M_dot_M(QLA_D_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_M_dot_M");
  qlab::api_reduce<qlab::DotOp<float, 4, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_M_dot_pM(QLA_D_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_M_dot_pM");
  qlab::api_reduce<qlab::DotOp<float, 4, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_pM_dot_M(QLA_D_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_pM_dot_M");
  qlab::api_reduce<qlab::DotOp<float, 4, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_veq_pM_dot_pM(QLA_D_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF2_c_veq_pM_dot_pM");
  qlab::api_reduce<qlab::DotOp<float, 4, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_M_dot_M(QLA_D_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_M_dot_M");
  qlab::api_reduce<qlab::DotOp<float, 4, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_M_dot_pM(QLA_D_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, QLA_F2_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_M_dot_pM");
  qlab::api_reduce<qlab::DotOp<float, 4, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_pM_dot_M(QLA_D_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_pM_dot_M");
  qlab::api_reduce<qlab::DotOp<float, 4, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF2_c_xeq_pM_dot_pM(QLA_D_Complex *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, QLA_F2_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF2_c_xeq_pM_dot_pM");
  qlab::api_reduce<qlab::DotOp<float, 4, double>>("F2_dot", r, 2 * sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

}  // extern "C"
