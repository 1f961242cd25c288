// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F3 convert entry points (extern "C"), reference: lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, QLA_FD_c_eq_c rounding)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_sitefield.cuh"

extern "C" {
QLAB_EXPORT void QLA_DF3_V_veq_V(QLA_D3_ColorVector *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF3_V_veq_V");
  qlab::api_convert<float, double, 3>("F3_convert", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_FD3_V_veq_V(QLA_F3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_FD3_V_veq_V");
  qlab::api_convert<double, float, 3>("F3_convert", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_V_veq_pV(QLA_D3_ColorVector *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF3_V_veq_pV");
  qlab::api_convert<float, double, 3>("F3_convert", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_FD3_V_veq_pV(QLA_F3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_FD3_V_veq_pV");
  qlab::api_convert<double, float, 3>("F3_convert", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_H_veq_H(QLA_D3_HalfFermion *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF3_H_veq_H");
  qlab::api_convert<float, double, 6>("F3_convert", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_FD3_H_veq_H(QLA_F3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_FD3_H_veq_H");
  qlab::api_convert<double, float, 6>("F3_convert", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_H_veq_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF3_H_veq_pH");
  qlab::api_convert<float, double, 6>("F3_convert", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_FD3_H_veq_pH(QLA_F3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_FD3_H_veq_pH");
  qlab::api_convert<double, float, 6>("F3_convert", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_D_veq_D(QLA_D3_DiracFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF3_D_veq_D");
  qlab::api_convert<float, double, 12>("F3_convert", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_FD3_D_veq_D(QLA_F3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_FD3_D_veq_D");
  qlab::api_convert<double, float, 12>("F3_convert", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_D_veq_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF3_D_veq_pD");
  qlab::api_convert<float, double, 12>("F3_convert", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_FD3_D_veq_pD(QLA_F3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_FD3_D_veq_pD");
  qlab::api_convert<double, float, 12>("F3_convert", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_M_veq_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF3_M_veq_M");
  qlab::api_convert<float, double, 9>("F3_convert", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_FD3_M_veq_M(QLA_F3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_FD3_M_veq_M");
  qlab::api_convert<double, float, 9>("F3_convert", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_M_veq_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF3_M_veq_pM");
  qlab::api_convert<float, double, 9>("F3_convert", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_FD3_M_veq_pM(QLA_F3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_FD3_M_veq_pM");
  qlab::api_convert<double, float, 9>("F3_convert", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_P_veq_P(QLA_D3_DiracPropagator *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF3_P_veq_P");
  qlab::api_convert<float, double, 144>("F3_convert", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_FD3_P_veq_P(QLA_F3_DiracPropagator *__restrict__ r, QLA_D3_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_FD3_P_veq_P");
  qlab::api_convert<double, float, 144>("F3_convert", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_P_veq_pP(QLA_D3_DiracPropagator *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF3_P_veq_pP");
  qlab::api_convert<float, double, 144>("F3_convert", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_FD3_P_veq_pP(QLA_F3_DiracPropagator *__restrict__ r, QLA_D3_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_FD3_P_veq_pP");
  qlab::api_convert<double, float, 144>("F3_convert", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_V_xeq_V(QLA_D3_ColorVector *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_V_xeq_V");
  qlab::api_convert<float, double, 3>("F3_convert", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_FD3_V_xeq_V(QLA_F3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_FD3_V_xeq_V");
  qlab::api_convert<double, float, 3>("F3_convert", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DF3_V_xeq_pV(QLA_D3_ColorVector *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_V_xeq_pV");
  qlab::api_convert<float, double, 3>("F3_convert", r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_FD3_V_xeq_pV(QLA_F3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_FD3_V_xeq_pV");
  qlab::api_convert<double, float, 3>("F3_convert", r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DF3_H_xeq_H(QLA_D3_HalfFermion *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_H_xeq_H");
  qlab::api_convert<float, double, 6>("F3_convert", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_FD3_H_xeq_H(QLA_F3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_FD3_H_xeq_H");
  qlab::api_convert<double, float, 6>("F3_convert", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DF3_H_xeq_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_H_xeq_pH");
  qlab::api_convert<float, double, 6>("F3_convert", r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_FD3_H_xeq_pH(QLA_F3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_FD3_H_xeq_pH");
  qlab::api_convert<double, float, 6>("F3_convert", r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DF3_D_xeq_D(QLA_D3_DiracFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_D_xeq_D");
  qlab::api_convert<float, double, 12>("F3_convert", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_FD3_D_xeq_D(QLA_F3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_FD3_D_xeq_D");
  qlab::api_convert<double, float, 12>("F3_convert", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DF3_D_xeq_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_D_xeq_pD");
  qlab::api_convert<float, double, 12>("F3_convert", r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_FD3_D_xeq_pD(QLA_F3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_FD3_D_xeq_pD");
  qlab::api_convert<double, float, 12>("F3_convert", r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DF3_M_xeq_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_M_xeq_M");
  qlab::api_convert<float, double, 9>("F3_convert", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_FD3_M_xeq_M(QLA_F3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_FD3_M_xeq_M");
  qlab::api_convert<double, float, 9>("F3_convert", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DF3_M_xeq_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_M_xeq_pM");
  qlab::api_convert<float, double, 9>("F3_convert", r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_FD3_M_xeq_pM(QLA_F3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_FD3_M_xeq_pM");
  qlab::api_convert<double, float, 9>("F3_convert", r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DF3_P_xeq_P(QLA_D3_DiracPropagator *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_P_xeq_P");
  qlab::api_convert<float, double, 144>("F3_convert", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_FD3_P_xeq_P(QLA_F3_DiracPropagator *__restrict__ r, QLA_D3_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_FD3_P_xeq_P");
  qlab::api_convert<double, float, 144>("F3_convert", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DF3_P_xeq_pP(QLA_D3_DiracPropagator *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_P_xeq_pP");
  qlab::api_convert<float, double, 144>("F3_convert", r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_FD3_P_xeq_pP(QLA_F3_DiracPropagator *__restrict__ r, QLA_D3_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_FD3_P_xeq_pP");
  qlab::api_convert<double, float, 144>("F3_convert", r, qlab::op_ptr((const void* const*)a), index, n);
}

}  // extern "C"
