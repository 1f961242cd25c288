// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA D2 gsum entry points (extern "C"), reference: lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_ncolor.cuh"
#include "../qla_random.cuh"

extern "C" {
QLAB_EXPORT void QLA_D2_v_veq_sum_V(QLA_D2_ColorVector *__restrict__ r, QLA_D2_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_v_veq_sum_V");
  qlab::api_gsum_n<double, double>("D2_gsum", 2, 2, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_D2_v_veq_sum_pV(QLA_D2_ColorVector *__restrict__ r, QLA_D2_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_v_veq_sum_pV");
  qlab::api_gsum_n<double, double>("D2_gsum", 2, 2, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_D2_h_veq_sum_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_h_veq_sum_H");
  qlab::api_gsum_n<double, double>("D2_gsum", 2, 2 * 2, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_D2_h_veq_sum_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_h_veq_sum_pH");
  qlab::api_gsum_n<double, double>("D2_gsum", 2, 2 * 2, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_D2_d_veq_sum_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_d_veq_sum_D");
  qlab::api_gsum_n<double, double>("D2_gsum", 2, 4 * 2, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_D2_d_veq_sum_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_d_veq_sum_pD");
  qlab::api_gsum_n<double, double>("D2_gsum", 2, 4 * 2, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_D2_m_veq_sum_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_m_veq_sum_M");
  qlab::api_gsum_n<double, double>("D2_gsum", 2, 2 * 2, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_D2_m_veq_sum_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_m_veq_sum_pM");
  qlab::api_gsum_n<double, double>("D2_gsum", 2, 2 * 2, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_D2_p_veq_sum_P(QLA_D2_DiracPropagator *__restrict__ r, QLA_D2_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_p_veq_sum_P");
  qlab::api_gsum_n<double, double>("D2_gsum", 2, 16 * 2 * 2, r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_D2_p_veq_sum_pP(QLA_D2_DiracPropagator *__restrict__ r, QLA_D2_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_p_veq_sum_pP");
  qlab::api_gsum_n<double, double>("D2_gsum", 2, 16 * 2 * 2, r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_D2_v_xeq_sum_V(QLA_D2_ColorVector *__restrict__ r, QLA_D2_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_v_xeq_sum_V");
  qlab::api_gsum_n<double, double>("D2_gsum", 2, 2, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_D2_v_xeq_sum_pV(QLA_D2_ColorVector *__restrict__ r, QLA_D2_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_v_xeq_sum_pV");
  qlab::api_gsum_n<double, double>("D2_gsum", 2, 2, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_D2_h_xeq_sum_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_h_xeq_sum_H");
  qlab::api_gsum_n<double, double>("D2_gsum", 2, 2 * 2, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_D2_h_xeq_sum_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_h_xeq_sum_pH");
  qlab::api_gsum_n<double, double>("D2_gsum", 2, 2 * 2, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_D2_d_xeq_sum_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_d_xeq_sum_D");
  qlab::api_gsum_n<double, double>("D2_gsum", 2, 4 * 2, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_D2_d_xeq_sum_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_d_xeq_sum_pD");
  qlab::api_gsum_n<double, double>("D2_gsum", 2, 4 * 2, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_D2_m_xeq_sum_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_m_xeq_sum_M");
  qlab::api_gsum_n<double, double>("D2_gsum", 2, 2 * 2, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_D2_m_xeq_sum_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D2_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_m_xeq_sum_pM");
  qlab::api_gsum_n<double, double>("D2_gsum", 2, 2 * 2, r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_D2_p_xeq_sum_P(QLA_D2_DiracPropagator *__restrict__ r, QLA_D2_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_p_xeq_sum_P");
  qlab::api_gsum_n<double, double>("D2_gsum", 2, 16 * 2 * 2, r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_D2_p_xeq_sum_pP(QLA_D2_DiracPropagator *__restrict__ r, QLA_D2_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_p_xeq_sum_pP");
  qlab::api_gsum_n<double, double>("D2_gsum", 2, 16 * 2 * 2, r, qlab::op_ptr((const void* const*)a), index, n);
}

}  // extern "C"
