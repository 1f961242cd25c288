// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F3 redot entry points (extern "C"), reference: lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"

extern "C" {
QLAB_EXPORT void QLA_F3_r_veq_re_V_dot_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_r_veq_re_V_dot_V");
  qlab::api_reduce<qlab::ReDotOp<float, 3, float>>("F3_redot_V", r, sizeof(float), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_veq_re_V_dot_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_r_veq_re_V_dot_pV");
  qlab::api_reduce<qlab::ReDotOp<float, 3, float>>("F3_redot_V", r, sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_veq_re_pV_dot_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_r_veq_re_pV_dot_V");
  qlab::api_reduce<qlab::ReDotOp<float, 3, float>>("F3_redot_V", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_veq_re_pV_dot_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_r_veq_re_pV_dot_pV");
  qlab::api_reduce<qlab::ReDotOp<float, 3, float>>("F3_redot_V", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_re_V_dot_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_re_V_dot_V");
  qlab::api_reduce<qlab::ReDotOp<float, 3, float>>("F3_redot_V", r, sizeof(float), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_re_V_dot_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_re_V_dot_pV");
  qlab::api_reduce<qlab::ReDotOp<float, 3, float>>("F3_redot_V", r, sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_re_pV_dot_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_re_pV_dot_V");
  qlab::api_reduce<qlab::ReDotOp<float, 3, float>>("F3_redot_V", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_re_pV_dot_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_re_pV_dot_pV");
  qlab::api_reduce<qlab::ReDotOp<float, 3, float>>("F3_redot_V", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F3_r_veq_re_H_dot_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_r_veq_re_H_dot_H");
  qlab::api_reduce<qlab::ReDotOp<float, 6, float>>("F3_redot_H", r, sizeof(float), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_veq_re_H_dot_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_r_veq_re_H_dot_pH");
  qlab::api_reduce<qlab::ReDotOp<float, 6, float>>("F3_redot_H", r, sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_veq_re_pH_dot_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_r_veq_re_pH_dot_H");
  qlab::api_reduce<qlab::ReDotOp<float, 6, float>>("F3_redot_H", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_veq_re_pH_dot_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_r_veq_re_pH_dot_pH");
  qlab::api_reduce<qlab::ReDotOp<float, 6, float>>("F3_redot_H", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_re_H_dot_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_re_H_dot_H");
  qlab::api_reduce<qlab::ReDotOp<float, 6, float>>("F3_redot_H", r, sizeof(float), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_re_H_dot_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_re_H_dot_pH");
  qlab::api_reduce<qlab::ReDotOp<float, 6, float>>("F3_redot_H", r, sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_re_pH_dot_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_re_pH_dot_H");
  qlab::api_reduce<qlab::ReDotOp<float, 6, float>>("F3_redot_H", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_re_pH_dot_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_re_pH_dot_pH");
  qlab::api_reduce<qlab::ReDotOp<float, 6, float>>("F3_redot_H", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F3_r_veq_re_D_dot_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_r_veq_re_D_dot_D");
  qlab::api_reduce<qlab::ReDotOp<float, 12, float>>("F3_redot_D", r, sizeof(float), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_veq_re_D_dot_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_r_veq_re_D_dot_pD");
  qlab::api_reduce<qlab::ReDotOp<float, 12, float>>("F3_redot_D", r, sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_veq_re_pD_dot_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_r_veq_re_pD_dot_D");
  qlab::api_reduce<qlab::ReDotOp<float, 12, float>>("F3_redot_D", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_veq_re_pD_dot_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_r_veq_re_pD_dot_pD");
  qlab::api_reduce<qlab::ReDotOp<float, 12, float>>("F3_redot_D", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_re_D_dot_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_re_D_dot_D");
  qlab::api_reduce<qlab::ReDotOp<float, 12, float>>("F3_redot_D", r, sizeof(float), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_re_D_dot_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_re_D_dot_pD");
  qlab::api_reduce<qlab::ReDotOp<float, 12, float>>("F3_redot_D", r, sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_re_pD_dot_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_re_pD_dot_D");
  qlab::api_reduce<qlab::ReDotOp<float, 12, float>>("F3_redot_D", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_re_pD_dot_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_re_pD_dot_pD");
  qlab::api_reduce<qlab::ReDotOp<float, 12, float>>("F3_redot_D", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F3_r_veq_re_M_dot_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_r_veq_re_M_dot_M");
  qlab::api_reduce<qlab::ReDotOp<float, 9, float>>("F3_redot_M", r, sizeof(float), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_veq_re_M_dot_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_r_veq_re_M_dot_pM");
  qlab::api_reduce<qlab::ReDotOp<float, 9, float>>("F3_redot_M", r, sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_veq_re_pM_dot_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F3_r_veq_re_pM_dot_M");
  qlab::api_reduce<qlab::ReDotOp<float, 9, float>>("F3_redot_M", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_veq_re_pM_dot_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F3_r_veq_re_pM_dot_pM");
  qlab::api_reduce<qlab::ReDotOp<float, 9, float>>("F3_redot_M", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_re_M_dot_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_re_M_dot_M");
  qlab::api_reduce<qlab::ReDotOp<float, 9, float>>("F3_redot_M", r, sizeof(float), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_re_M_dot_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_re_M_dot_pM");
  qlab::api_reduce<qlab::ReDotOp<float, 9, float>>("F3_redot_M", r, sizeof(float), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_re_pM_dot_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_re_pM_dot_M");
  qlab::api_reduce<qlab::ReDotOp<float, 9, float>>("F3_redot_M", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_re_pM_dot_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_re_pM_dot_pM");
  qlab::api_reduce<qlab::ReDotOp<float, 9, float>>("F3_redot_M", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_re_V_dot_V(QLA_D_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_re_V_dot_V");
  qlab::api_reduce<qlab::ReDotOp<float, 3, double>>("F3_redot_V", r, sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_re_V_dot_pV(QLA_D_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_re_V_dot_pV");
  qlab::api_reduce<qlab::ReDotOp<float, 3, double>>("F3_redot_V", r, sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_re_pV_dot_V(QLA_D_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_re_pV_dot_V");
  qlab::api_reduce<qlab::ReDotOp<float, 3, double>>("F3_redot_V", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_re_pV_dot_pV(QLA_D_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_re_pV_dot_pV");
  qlab::api_reduce<qlab::ReDotOp<float, 3, double>>("F3_redot_V", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_re_V_dot_V(QLA_D_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_re_V_dot_V");
  qlab::api_reduce<qlab::ReDotOp<float, 3, double>>("F3_redot_V", r, sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_re_V_dot_pV(QLA_D_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_re_V_dot_pV");
  qlab::api_reduce<qlab::ReDotOp<float, 3, double>>("F3_redot_V", r, sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_re_pV_dot_V(QLA_D_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_re_pV_dot_V");
  qlab::api_reduce<qlab::ReDotOp<float, 3, double>>("F3_redot_V", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_re_pV_dot_pV(QLA_D_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, QLA_F3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_re_pV_dot_pV");
  qlab::api_reduce<qlab::ReDotOp<float, 3, double>>("F3_redot_V", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_re_H_dot_H(QLA_D_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_re_H_dot_H");
  qlab::api_reduce<qlab::ReDotOp<float, 6, double>>("F3_redot_H", r, sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_re_H_dot_pH(QLA_D_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_re_H_dot_pH");
  qlab::api_reduce<qlab::ReDotOp<float, 6, double>>("F3_redot_H", r, sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_re_pH_dot_H(QLA_D_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_re_pH_dot_H");
  qlab::api_reduce<qlab::ReDotOp<float, 6, double>>("F3_redot_H", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_re_pH_dot_pH(QLA_D_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_re_pH_dot_pH");
  qlab::api_reduce<qlab::ReDotOp<float, 6, double>>("F3_redot_H", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_re_H_dot_H(QLA_D_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_re_H_dot_H");
  qlab::api_reduce<qlab::ReDotOp<float, 6, double>>("F3_redot_H", r, sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_re_H_dot_pH(QLA_D_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, QLA_F3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_re_H_dot_pH");
  qlab::api_reduce<qlab::ReDotOp<float, 6, double>>("F3_redot_H", r, sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_re_pH_dot_H(QLA_D_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_re_pH_dot_H");
  qlab::api_reduce<qlab::ReDotOp<float, 6, double>>("F3_redot_H", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_re_pH_dot_pH(QLA_D_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, QLA_F3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_re_pH_dot_pH");
  qlab::api_reduce<qlab::ReDotOp<float, 6, double>>("F3_redot_H", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_re_D_dot_D(QLA_D_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_re_D_dot_D");
  qlab::api_reduce<qlab::ReDotOp<float, 12, double>>("F3_redot_D", r, sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_re_D_dot_pD(QLA_D_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_re_D_dot_pD");
  qlab::api_reduce<qlab::ReDotOp<float, 12, double>>("F3_redot_D", r, sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_re_pD_dot_D(QLA_D_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_re_pD_dot_D");
  qlab::api_reduce<qlab::ReDotOp<float, 12, double>>("F3_redot_D", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_re_pD_dot_pD(QLA_D_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_re_pD_dot_pD");
  qlab::api_reduce<qlab::ReDotOp<float, 12, double>>("F3_redot_D", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_re_D_dot_D(QLA_D_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_re_D_dot_D");
  qlab::api_reduce<qlab::ReDotOp<float, 12, double>>("F3_redot_D", r, sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_re_D_dot_pD(QLA_D_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, QLA_F3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_re_D_dot_pD");
  qlab::api_reduce<qlab::ReDotOp<float, 12, double>>("F3_redot_D", r, sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_re_pD_dot_D(QLA_D_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_re_pD_dot_D");
  qlab::api_reduce<qlab::ReDotOp<float, 12, double>>("F3_redot_D", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_re_pD_dot_pD(QLA_D_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, QLA_F3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_re_pD_dot_pD");
  qlab::api_reduce<qlab::ReDotOp<float, 12, double>>("F3_redot_D", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_re_M_dot_M(QLA_D_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_re_M_dot_M");
  qlab::api_reduce<qlab::ReDotOp<float, 9, double>>("F3_redot_M", r, sizeof(double), qlab::op_contig(a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_re_M_dot_pM(QLA_D_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_re_M_dot_pM");
  qlab::api_reduce<qlab::ReDotOp<float, 9, double>>("F3_redot_M", r, sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_re_pM_dot_M(QLA_D_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_re_pM_dot_M");
  qlab::api_reduce<qlab::ReDotOp<float, 9, double>>("F3_redot_M", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_re_pM_dot_pM(QLA_D_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_re_pM_dot_pM");
  qlab::api_reduce<qlab::ReDotOp<float, 9, double>>("F3_redot_M", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_re_M_dot_M(QLA_D_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_re_M_dot_M");
  qlab::api_reduce<qlab::ReDotOp<float, 9, double>>("F3_redot_M", r, sizeof(double), qlab::op_contig(a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_re_M_dot_pM(QLA_D_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_re_M_dot_pM");
  qlab::api_reduce<qlab::ReDotOp<float, 9, double>>("F3_redot_M", r, sizeof(double), qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_re_pM_dot_M(QLA_D_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_re_pM_dot_M");
  qlab::api_reduce<qlab::ReDotOp<float, 9, double>>("F3_redot_M", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_re_pM_dot_pM(QLA_D_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, QLA_F3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_re_pM_dot_pM");
  qlab::api_reduce<qlab::ReDotOp<float, 9, double>>("F3_redot_M", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n);
}

}  // extern "C"
