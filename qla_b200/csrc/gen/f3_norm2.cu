// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F3 norm2 entry points (extern "C"), reference: lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"

extern "C" {
QLAB_EXPORT void QLA_F3_r_veq_norm2_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_r_veq_norm2_V");
  qlab::api_reduce<qlab::Norm2Op<float, 3, float>>("F3_norm2_V", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_veq_norm2_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_r_veq_norm2_pV");
  qlab::api_reduce<qlab::Norm2Op<float, 3, float>>("F3_norm2_V", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_norm2_V(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_norm2_V");
  qlab::api_reduce<qlab::Norm2Op<float, 3, float>>("F3_norm2_V", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_norm2_pV(QLA_F_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_norm2_pV");
  qlab::api_reduce<qlab::Norm2Op<float, 3, float>>("F3_norm2_V", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_F3_r_veq_norm2_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_r_veq_norm2_H");
  qlab::api_reduce<qlab::Norm2Op<float, 6, float>>("F3_norm2_H", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_veq_norm2_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_r_veq_norm2_pH");
  qlab::api_reduce<qlab::Norm2Op<float, 6, float>>("F3_norm2_H", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_norm2_H(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_norm2_H");
  qlab::api_reduce<qlab::Norm2Op<float, 6, float>>("F3_norm2_H", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_norm2_pH(QLA_F_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_norm2_pH");
  qlab::api_reduce<qlab::Norm2Op<float, 6, float>>("F3_norm2_H", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_F3_r_veq_norm2_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_r_veq_norm2_D");
  qlab::api_reduce<qlab::Norm2Op<float, 12, float>>("F3_norm2_D", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_veq_norm2_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_r_veq_norm2_pD");
  qlab::api_reduce<qlab::Norm2Op<float, 12, float>>("F3_norm2_D", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_norm2_D(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_norm2_D");
  qlab::api_reduce<qlab::Norm2Op<float, 12, float>>("F3_norm2_D", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_norm2_pD(QLA_F_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_norm2_pD");
  qlab::api_reduce<qlab::Norm2Op<float, 12, float>>("F3_norm2_D", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_F3_r_veq_norm2_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_r_veq_norm2_M");
  qlab::api_reduce<qlab::Norm2Op<float, 9, float>>("F3_norm2_M", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_veq_norm2_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_r_veq_norm2_pM");
  qlab::api_reduce<qlab::Norm2Op<float, 9, float>>("F3_norm2_M", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_norm2_M(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_norm2_M");
  qlab::api_reduce<qlab::Norm2Op<float, 9, float>>("F3_norm2_M", r, sizeof(float), qlab::op_contig(a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_F3_r_xeq_norm2_pM(QLA_F_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_r_xeq_norm2_pM");
  qlab::api_reduce<qlab::Norm2Op<float, 9, float>>("F3_norm2_M", r, sizeof(float), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_norm2_V(QLA_D_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_norm2_V");
  qlab::api_reduce<qlab::Norm2Op<float, 3, double>>("F3_norm2_V", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_norm2_pV(QLA_D_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_norm2_pV");
  qlab::api_reduce<qlab::Norm2Op<float, 3, double>>("F3_norm2_V", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_norm2_V(QLA_D_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_norm2_V");
  qlab::api_reduce<qlab::Norm2Op<float, 3, double>>("F3_norm2_V", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_norm2_pV(QLA_D_Real *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_norm2_pV");
  qlab::api_reduce<qlab::Norm2Op<float, 3, double>>("F3_norm2_V", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_norm2_H(QLA_D_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_norm2_H");
  qlab::api_reduce<qlab::Norm2Op<float, 6, double>>("F3_norm2_H", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_norm2_pH(QLA_D_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_norm2_pH");
  qlab::api_reduce<qlab::Norm2Op<float, 6, double>>("F3_norm2_H", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_norm2_H(QLA_D_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_norm2_H");
  qlab::api_reduce<qlab::Norm2Op<float, 6, double>>("F3_norm2_H", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_norm2_pH(QLA_D_Real *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_norm2_pH");
  qlab::api_reduce<qlab::Norm2Op<float, 6, double>>("F3_norm2_H", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_norm2_D(QLA_D_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_norm2_D");
  qlab::api_reduce<qlab::Norm2Op<float, 12, double>>("F3_norm2_D", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_norm2_pD(QLA_D_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_norm2_pD");
  qlab::api_reduce<qlab::Norm2Op<float, 12, double>>("F3_norm2_D", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_norm2_D(QLA_D_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_norm2_D");
  qlab::api_reduce<qlab::Norm2Op<float, 12, double>>("F3_norm2_D", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_norm2_pD(QLA_D_Real *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_norm2_pD");
  qlab::api_reduce<qlab::Norm2Op<float, 12, double>>("F3_norm2_D", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_norm2_M(QLA_D_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_norm2_M");
  qlab::api_reduce<qlab::Norm2Op<float, 9, double>>("F3_norm2_M", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_veq_norm2_pM(QLA_D_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF3_r_veq_norm2_pM");
  qlab::api_reduce<qlab::Norm2Op<float, 9, double>>("F3_norm2_M", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_norm2_M(QLA_D_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_norm2_M");
  qlab::api_reduce<qlab::Norm2Op<float, 9, double>>("F3_norm2_M", r, sizeof(double), qlab::op_contig(a), qlab::Opnd{}, index, n);
}

QLAB_EXPORT void QLA_DF3_r_xeq_norm2_pM(QLA_D_Real *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_r_xeq_norm2_pM");
  qlab::api_reduce<qlab::Norm2Op<float, 9, double>>("F3_norm2_M", r, sizeof(double), qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n);
}

}  // extern "C"
