// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA D2 rtimes entry points (extern "C"), reference: lib/perl/build_qla.pl:1256-1292 (real constant times field)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"

extern "C" {
QLAB_EXPORT void QLA_D2_V_veq_r_times_V(QLA_D2_ColorVector *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_V_veq_r_times_V");
  qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_V_veq_r_times_pV(QLA_D2_ColorVector *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_V_veq_r_times_pV");
  qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_V_vpeq_r_times_V(QLA_D2_ColorVector *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_V_vpeq_r_times_V");
  qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_V_vpeq_r_times_pV(QLA_D2_ColorVector *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_V_vpeq_r_times_pV");
  qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_V_vmeq_r_times_V(QLA_D2_ColorVector *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_V_vmeq_r_times_V");
  qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_V_vmeq_r_times_pV(QLA_D2_ColorVector *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_V_vmeq_r_times_pV");
  qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_V_veqm_r_times_V(QLA_D2_ColorVector *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_V_veqm_r_times_V");
  qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_V_veqm_r_times_pV(QLA_D2_ColorVector *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_V_veqm_r_times_pV");
  qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_V_xeq_r_times_V(QLA_D2_ColorVector *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_V_xeq_r_times_V");
  qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_V_xeq_r_times_pV(QLA_D2_ColorVector *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_V_xeq_r_times_pV");
  qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_V_xpeq_r_times_V(QLA_D2_ColorVector *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_V_xpeq_r_times_V");
  qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_V_xpeq_r_times_pV(QLA_D2_ColorVector *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_V_xpeq_r_times_pV");
  qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_V_xmeq_r_times_V(QLA_D2_ColorVector *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_V_xmeq_r_times_V");
  qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_V_xmeq_r_times_pV(QLA_D2_ColorVector *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_V_xmeq_r_times_pV");
  qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_V_xeqm_r_times_V(QLA_D2_ColorVector *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_V_xeqm_r_times_V");
  qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_V_xeqm_r_times_pV(QLA_D2_ColorVector *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_V_xeqm_r_times_pV");
  qlab::api_scalar_map<qlab::RTimesOp<double, 2>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_veq_r_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_r_times_H");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_r_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_r_times_pH");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_vpeq_r_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_vpeq_r_times_H");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_vpeq_r_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_vpeq_r_times_pH");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_vmeq_r_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_vmeq_r_times_H");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_vmeq_r_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_vmeq_r_times_pH");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_veqm_r_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_veqm_r_times_H");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_veqm_r_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_veqm_r_times_pH");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_xeq_r_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_r_times_H");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_r_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_r_times_pH");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xpeq_r_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xpeq_r_times_H");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_xpeq_r_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xpeq_r_times_pH");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_xmeq_r_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xmeq_r_times_H");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_xmeq_r_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xmeq_r_times_pH");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_xeqm_r_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeqm_r_times_H");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_xeqm_r_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeqm_r_times_pH");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_veq_r_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_r_times_D");
  qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_r_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_r_times_pD");
  qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_vpeq_r_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_vpeq_r_times_D");
  qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_vpeq_r_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_vpeq_r_times_pD");
  qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_vmeq_r_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_vmeq_r_times_D");
  qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_vmeq_r_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_vmeq_r_times_pD");
  qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_veqm_r_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_veqm_r_times_D");
  qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_veqm_r_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_veqm_r_times_pD");
  qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_xeq_r_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_r_times_D");
  qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_r_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_r_times_pD");
  qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xpeq_r_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xpeq_r_times_D");
  qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_xpeq_r_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xpeq_r_times_pD");
  qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_xmeq_r_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xmeq_r_times_D");
  qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_xmeq_r_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xmeq_r_times_pD");
  qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_xeqm_r_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeqm_r_times_D");
  qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_xeqm_r_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeqm_r_times_pD");
  qlab::api_scalar_map<qlab::RTimesOp<double, 8>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_M_veq_r_times_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_M_veq_r_times_M");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_veq_r_times_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_M_veq_r_times_pM");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_vpeq_r_times_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_M_vpeq_r_times_M");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_M_vpeq_r_times_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_M_vpeq_r_times_pM");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_M_vmeq_r_times_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_M_vmeq_r_times_M");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_M_vmeq_r_times_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_M_vmeq_r_times_pM");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_M_veqm_r_times_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_M_veqm_r_times_M");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_M_veqm_r_times_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_M_veqm_r_times_pM");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_M_xeq_r_times_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xeq_r_times_M");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_xeq_r_times_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xeq_r_times_pM");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_M_xpeq_r_times_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xpeq_r_times_M");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_M_xpeq_r_times_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xpeq_r_times_pM");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_M_xmeq_r_times_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xmeq_r_times_M");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_M_xmeq_r_times_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xmeq_r_times_pM");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_M_xeqm_r_times_M(QLA_D2_ColorMatrix *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xeqm_r_times_M");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_M_xeqm_r_times_pM(QLA_D2_ColorMatrix *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_M_xeqm_r_times_pM");
  qlab::api_scalar_map<qlab::RTimesOp<double, 4>, double>("D2_rtimes", r, (const double*)a, qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

}  // extern "C"
