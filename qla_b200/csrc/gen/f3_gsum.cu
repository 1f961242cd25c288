// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F3 gsum entry points (extern "C"), reference: lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_sitefield.cuh"

extern "C" {
QLAB_EXPORT void QLA_F3_v_veq_sum_V(QLA_F3_ColorVector *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_v_veq_sum_V");
  qlab::api_gsum<float, 3>("F3_gsum", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_F3_v_veq_sum_pV(QLA_F3_ColorVector *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_v_veq_sum_pV");
  qlab::api_gsum<float, 3>("F3_gsum", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_F3_h_veq_sum_H(QLA_F3_HalfFermion *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_h_veq_sum_H");
  qlab::api_gsum<float, 6>("F3_gsum", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_F3_h_veq_sum_pH(QLA_F3_HalfFermion *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_h_veq_sum_pH");
  qlab::api_gsum<float, 6>("F3_gsum", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_F3_d_veq_sum_D(QLA_F3_DiracFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_d_veq_sum_D");
  qlab::api_gsum<float, 12>("F3_gsum", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_F3_d_veq_sum_pD(QLA_F3_DiracFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_d_veq_sum_pD");
  qlab::api_gsum<float, 12>("F3_gsum", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_F3_m_veq_sum_M(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_m_veq_sum_M");
  qlab::api_gsum<float, 9>("F3_gsum", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_F3_m_veq_sum_pM(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_m_veq_sum_pM");
  qlab::api_gsum<float, 9>("F3_gsum", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_F3_p_veq_sum_P(QLA_F3_DiracPropagator *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F3_p_veq_sum_P");
  qlab::api_gsum<float, 144>("F3_gsum", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_F3_p_veq_sum_pP(QLA_F3_DiracPropagator *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F3_p_veq_sum_pP");
  qlab::api_gsum<float, 144>("F3_gsum", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_v_veq_sum_V(QLA_D3_ColorVector *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF3_v_veq_sum_V");
  qlab::api_gsum<float, 3, double>("F3_gsum_df", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_v_veq_sum_pV(QLA_D3_ColorVector *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF3_v_veq_sum_pV");
  qlab::api_gsum<float, 3, double>("F3_gsum_df", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_h_veq_sum_H(QLA_D3_HalfFermion *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF3_h_veq_sum_H");
  qlab::api_gsum<float, 6, double>("F3_gsum_df", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_h_veq_sum_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF3_h_veq_sum_pH");
  qlab::api_gsum<float, 6, double>("F3_gsum_df", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_d_veq_sum_D(QLA_D3_DiracFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF3_d_veq_sum_D");
  qlab::api_gsum<float, 12, double>("F3_gsum_df", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_d_veq_sum_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF3_d_veq_sum_pD");
  qlab::api_gsum<float, 12, double>("F3_gsum_df", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_m_veq_sum_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF3_m_veq_sum_M");
  qlab::api_gsum<float, 9, double>("F3_gsum_df", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_m_veq_sum_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF3_m_veq_sum_pM");
  qlab::api_gsum<float, 9, double>("F3_gsum_df", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_p_veq_sum_P(QLA_D3_DiracPropagator *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, int n) {
  QLAB_TRACE("QLA_DF3_p_veq_sum_P");
  qlab::api_gsum<float, 144, double>("F3_gsum_df", r, qlab::op_contig(a), nullptr, n);
}

QLAB_EXPORT void QLA_DF3_p_veq_sum_pP(QLA_D3_DiracPropagator *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_DF3_p_veq_sum_pP");
  qlab::api_gsum<float, 144, double>("F3_gsum_df", r, qlab::op_ptr((const void* const*)a), nullptr, n);
}

QLAB_EXPORT void QLA_F3_v_xeq_sum_V(QLA_F3_ColorVector *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_v_xeq_sum_V");
  qlab::api_gsum<float, 3>("F3_gsum", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_F3_v_xeq_sum_pV(QLA_F3_ColorVector *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_v_xeq_sum_pV");
  qlab::api_gsum<float, 3>("F3_gsum", r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_F3_h_xeq_sum_H(QLA_F3_HalfFermion *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_h_xeq_sum_H");
  qlab::api_gsum<float, 6>("F3_gsum", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_F3_h_xeq_sum_pH(QLA_F3_HalfFermion *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_h_xeq_sum_pH");
  qlab::api_gsum<float, 6>("F3_gsum", r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_F3_d_xeq_sum_D(QLA_F3_DiracFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_d_xeq_sum_D");
  qlab::api_gsum<float, 12>("F3_gsum", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_F3_d_xeq_sum_pD(QLA_F3_DiracFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_d_xeq_sum_pD");
  qlab::api_gsum<float, 12>("F3_gsum", r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_F3_m_xeq_sum_M(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_m_xeq_sum_M");
  qlab::api_gsum<float, 9>("F3_gsum", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_F3_m_xeq_sum_pM(QLA_F3_ColorMatrix *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_m_xeq_sum_pM");
  qlab::api_gsum<float, 9>("F3_gsum", r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_F3_p_xeq_sum_P(QLA_F3_DiracPropagator *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F3_p_xeq_sum_P");
  qlab::api_gsum<float, 144>("F3_gsum", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_F3_p_xeq_sum_pP(QLA_F3_DiracPropagator *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F3_p_xeq_sum_pP");
  qlab::api_gsum<float, 144>("F3_gsum", r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DF3_v_xeq_sum_V(QLA_D3_ColorVector *__restrict__ r, QLA_F3_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_v_xeq_sum_V");
  qlab::api_gsum<float, 3, double>("F3_gsum_df", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DF3_v_xeq_sum_pV(QLA_D3_ColorVector *__restrict__ r, QLA_F3_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_v_xeq_sum_pV");
  qlab::api_gsum<float, 3, double>("F3_gsum_df", r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DF3_h_xeq_sum_H(QLA_D3_HalfFermion *__restrict__ r, QLA_F3_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_h_xeq_sum_H");
  qlab::api_gsum<float, 6, double>("F3_gsum_df", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DF3_h_xeq_sum_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_F3_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_h_xeq_sum_pH");
  qlab::api_gsum<float, 6, double>("F3_gsum_df", r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DF3_d_xeq_sum_D(QLA_D3_DiracFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_d_xeq_sum_D");
  qlab::api_gsum<float, 12, double>("F3_gsum_df", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DF3_d_xeq_sum_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_d_xeq_sum_pD");
  qlab::api_gsum<float, 12, double>("F3_gsum_df", r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DF3_m_xeq_sum_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_m_xeq_sum_M");
  qlab::api_gsum<float, 9, double>("F3_gsum_df", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DF3_m_xeq_sum_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_F3_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_m_xeq_sum_pM");
  qlab::api_gsum<float, 9, double>("F3_gsum_df", r, qlab::op_ptr((const void* const*)a), index, n);
}

QLAB_EXPORT void QLA_DF3_p_xeq_sum_P(QLA_D3_DiracPropagator *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_p_xeq_sum_P");
  qlab::api_gsum<float, 144, double>("F3_gsum_df", r, qlab::op_contig(a), index, n);
}

QLAB_EXPORT void QLA_DF3_p_xeq_sum_pP(QLA_D3_DiracPropagator *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_DF3_p_xeq_sum_pP");
  qlab::api_gsum<float, 144, double>("F3_gsum_df", r, qlab::op_ptr((const void* const*)a), index, n);
}

}  // extern "C"
