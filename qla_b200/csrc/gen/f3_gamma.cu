// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F3 gamma entry points (extern "C"), reference: lib/perl/build_qla.pl:1358-1412 (left / right multiplication by gamma_mu, mu = 0..15), expressions_gamma.pl:59-134, 384-470
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_sitefield.cuh"

extern "C" {
QLAB_EXPORT void QLA_F3_D_veq_gamma_times_D(QLA_F3_DiracFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int mu, int n) {
  QLAB_TRACE("QLA_F3_D_veq_gamma_times_D");
  qlab::api_gamma<float, 12, true>("F3_gamma", r, qlab::op_contig(a), mu, nullptr, n);
}

QLAB_EXPORT void QLA_F3_D_veq_gamma_times_pD(QLA_F3_DiracFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int mu, int n) {
  QLAB_TRACE("QLA_F3_D_veq_gamma_times_pD");
  qlab::api_gamma<float, 12, true>("F3_gamma", r, qlab::op_ptr((const void* const*)a), mu, nullptr, n);
}

QLAB_EXPORT void QLA_F3_P_veq_gamma_times_P(QLA_F3_DiracPropagator *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, int mu, int n) {
  QLAB_TRACE("QLA_F3_P_veq_gamma_times_P");
  qlab::api_gamma<float, 144, true>("F3_gamma", r, qlab::op_contig(a), mu, nullptr, n);
}

QLAB_EXPORT void QLA_F3_P_veq_gamma_times_pP(QLA_F3_DiracPropagator *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, int mu, int n) {
  QLAB_TRACE("QLA_F3_P_veq_gamma_times_pP");
  qlab::api_gamma<float, 144, true>("F3_gamma", r, qlab::op_ptr((const void* const*)a), mu, nullptr, n);
}

QLAB_EXPORT void QLA_F3_P_veq_P_times_gamma(QLA_F3_DiracPropagator *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, int mu, int n) {
  QLAB_TRACE("QLA_F3_P_veq_P_times_gamma");
  qlab::api_gamma<float, 144, false>("F3_gamma", r, qlab::op_contig(a), mu, nullptr, n);
}

QLAB_EXPORT void QLA_F3_P_veq_pP_times_gamma(QLA_F3_DiracPropagator *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, int mu, int n) {
  QLAB_TRACE("QLA_F3_P_veq_pP_times_gamma");
  qlab::api_gamma<float, 144, false>("F3_gamma", r, qlab::op_ptr((const void* const*)a), mu, nullptr, n);
}

QLAB_EXPORT void QLA_F3_D_xeq_gamma_times_D(QLA_F3_DiracFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int mu, int * index, int n) {
  QLAB_TRACE("QLA_F3_D_xeq_gamma_times_D");
  qlab::api_gamma<float, 12, true>("F3_gamma", r, qlab::op_contig(a), mu, index, n);
}

QLAB_EXPORT void QLA_F3_D_xeq_gamma_times_pD(QLA_F3_DiracFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int mu, int * index, int n) {
  QLAB_TRACE("QLA_F3_D_xeq_gamma_times_pD");
  qlab::api_gamma<float, 12, true>("F3_gamma", r, qlab::op_ptr((const void* const*)a), mu, index, n);
}

QLAB_EXPORT void QLA_F3_P_xeq_gamma_times_P(QLA_F3_DiracPropagator *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, int mu, int * index, int n) {
  QLAB_TRACE("QLA_F3_P_xeq_gamma_times_P");
  qlab::api_gamma<float, 144, true>("F3_gamma", r, qlab::op_contig(a), mu, index, n);
}

QLAB_EXPORT void QLA_F3_P_xeq_gamma_times_pP(QLA_F3_DiracPropagator *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, int mu, int * index, int n) {
  QLAB_TRACE("QLA_F3_P_xeq_gamma_times_pP");
  qlab::api_gamma<float, 144, true>("F3_gamma", r, qlab::op_ptr((const void* const*)a), mu, index, n);
}

QLAB_EXPORT void QLA_F3_P_xeq_P_times_gamma(QLA_F3_DiracPropagator *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ a, int mu, int * index, int n) {
  QLAB_TRACE("QLA_F3_P_xeq_P_times_gamma");
  qlab::api_gamma<float, 144, false>("F3_gamma", r, qlab::op_contig(a), mu, index, n);
}

QLAB_EXPORT void QLA_F3_P_xeq_pP_times_gamma(QLA_F3_DiracPropagator *__restrict__ r, QLA_F3_DiracPropagator *__restrict__ * a, int mu, int * index, int n) {
  QLAB_TRACE("QLA_F3_P_xeq_pP_times_gamma");
  qlab::api_gamma<float, 144, false>("F3_gamma", r, qlab::op_ptr((const void* const*)a), mu, index, n);
}

}  // extern "C"
