// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F2 convert entry points (extern "C"), reference: lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_ncolor.cuh"
#include "../qla_random.cuh"

extern "C" {
QLAB_EXPORT void QLA_DF2_V_veq_V(QLA_D2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF2_V_veq_V");
  qlab::api_convert_n<float, double>("F2_convert", 2, 2, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_FD2_V_veq_V(QLA_F2_ColorVector *__restrict__ r, QLA_D2_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_FD2_V_veq_V");
  qlab::api_convert_n<double, float>("F2_convert", 2, 2, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_V_veq_pV(QLA_D2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF2_V_veq_pV");
  qlab::api_convert_n<float, double>("F2_convert", 2, 2, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_FD2_V_veq_pV(QLA_F2_ColorVector *__restrict__ r, QLA_D2_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_FD2_V_veq_pV");
  qlab::api_convert_n<double, float>("F2_convert", 2, 2, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_H_veq_H(QLA_D2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF2_H_veq_H");
  qlab::api_convert_n<float, double>("F2_convert", 2, 2 * 2, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_FD2_H_veq_H(QLA_F2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_FD2_H_veq_H");
  qlab::api_convert_n<double, float>("F2_convert", 2, 2 * 2, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_H_veq_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF2_H_veq_pH");
  qlab::api_convert_n<float, double>("F2_convert", 2, 2 * 2, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_FD2_H_veq_pH(QLA_F2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_FD2_H_veq_pH");
  qlab::api_convert_n<double, float>("F2_convert", 2, 2 * 2, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_D_veq_D(QLA_D2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF2_D_veq_D");
  qlab::api_convert_n<float, double>("F2_convert", 2, 4 * 2, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_FD2_D_veq_D(QLA_F2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_FD2_D_veq_D");
  qlab::api_convert_n<double, float>("F2_convert", 2, 4 * 2, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_D_veq_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF2_D_veq_pD");
  qlab::api_convert_n<float, double>("F2_convert", 2, 4 * 2, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_FD2_D_veq_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_FD2_D_veq_pD");
  qlab::api_convert_n<double, float>("F2_convert", 2, 4 * 2, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_M_veq_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF2_M_veq_M");
  qlab::api_convert_n<float, double>("F2_convert", 2, 2 * 2, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_FD2_M_veq_M(QLA_F2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_FD2_M_veq_M");
  qlab::api_convert_n<double, float>("F2_convert", 2, 2 * 2, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_M_veq_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF2_M_veq_pM");
  qlab::api_convert_n<float, double>("F2_convert", 2, 2 * 2, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_FD2_M_veq_pM(QLA_F2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_FD2_M_veq_pM");
  qlab::api_convert_n<double, float>("F2_convert", 2, 2 * 2, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_P_veq_P(QLA_D2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF2_P_veq_P");
  qlab::api_convert_n<float, double>("F2_convert", 2, 16 * 2 * 2, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_FD2_P_veq_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_D2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_FD2_P_veq_P");
  qlab::api_convert_n<double, float>("F2_convert", 2, 16 * 2 * 2, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_P_veq_pP(QLA_D2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF2_P_veq_pP");
  qlab::api_convert_n<float, double>("F2_convert", 2, 16 * 2 * 2, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_FD2_P_veq_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_D2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_FD2_P_veq_pP");
  qlab::api_convert_n<double, float>("F2_convert", 2, 16 * 2 * 2, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DF2_V_xeq_V(QLA_D2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF2_V_xeq_V");
  qlab::api_convert_n<float, double>("F2_convert", 2, 2, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_FD2_V_xeq_V(QLA_F2_ColorVector *__restrict__ r, QLA_D2_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_FD2_V_xeq_V");
  qlab::api_convert_n<double, float>("F2_convert", 2, 2, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DF2_V_xeq_pV(QLA_D2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF2_V_xeq_pV");
  qlab::api_convert_n<float, double>("F2_convert", 2, 2, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_FD2_V_xeq_pV(QLA_F2_ColorVector *__restrict__ r, QLA_D2_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_FD2_V_xeq_pV");
  qlab::api_convert_n<double, float>("F2_convert", 2, 2, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DF2_H_xeq_H(QLA_D2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF2_H_xeq_H");
  qlab::api_convert_n<float, double>("F2_convert", 2, 2 * 2, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_FD2_H_xeq_H(QLA_F2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_FD2_H_xeq_H");
  qlab::api_convert_n<double, float>("F2_convert", 2, 2 * 2, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DF2_H_xeq_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF2_H_xeq_pH");
  qlab::api_convert_n<float, double>("F2_convert", 2, 2 * 2, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_FD2_H_xeq_pH(QLA_F2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_FD2_H_xeq_pH");
  qlab::api_convert_n<double, float>("F2_convert", 2, 2 * 2, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DF2_D_xeq_D(QLA_D2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF2_D_xeq_D");
  qlab::api_convert_n<float, double>("F2_convert", 2, 4 * 2, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_FD2_D_xeq_D(QLA_F2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_FD2_D_xeq_D");
  qlab::api_convert_n<double, float>("F2_convert", 2, 4 * 2, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DF2_D_xeq_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF2_D_xeq_pD");
  qlab::api_convert_n<float, double>("F2_convert", 2, 4 * 2, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_FD2_D_xeq_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_FD2_D_xeq_pD");
  qlab::api_convert_n<double, float>("F2_convert", 2, 4 * 2, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DF2_M_xeq_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF2_M_xeq_M");
  qlab::api_convert_n<float, double>("F2_convert", 2, 2 * 2, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_FD2_M_xeq_M(QLA_F2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_FD2_M_xeq_M");
  qlab::api_convert_n<double, float>("F2_convert", 2, 2 * 2, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DF2_M_xeq_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF2_M_xeq_pM");
  qlab::api_convert_n<float, double>("F2_convert", 2, 2 * 2, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_FD2_M_xeq_pM(QLA_F2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_FD2_M_xeq_pM");
  qlab::api_convert_n<double, float>("F2_convert", 2, 2 * 2, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DF2_P_xeq_P(QLA_D2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF2_P_xeq_P");
  qlab::api_convert_n<float, double>("F2_convert", 2, 16 * 2 * 2, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_FD2_P_xeq_P(QLA_F2_DiracPropagator *__restrict__ r, QLA_D2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_FD2_P_xeq_P");
  qlab::api_convert_n<double, float>("F2_convert", 2, 16 * 2 * 2, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DF2_P_xeq_pP(QLA_D2_DiracPropagator *__restrict__ r, QLA_F2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF2_P_xeq_pP");
  qlab::api_convert_n<float, double>("F2_convert", 2, 16 * 2 * 2, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_FD2_P_xeq_pP(QLA_F2_DiracPropagator *__restrict__ r, QLA_D2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_FD2_P_xeq_pP");
  qlab::api_convert_n<double, float>("F2_convert", 2, 16 * 2 * 2, r, qlab::op_ptr((const void* const*)a), index, n);
}

}  // extern "C"
