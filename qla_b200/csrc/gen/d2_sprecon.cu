// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA D2 sprecon entry points (extern "C"), reference: lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"

extern "C" {
QLAB_EXPORT void QLA_D2_D_veq_sprecon_H(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_D2_D_veq_sprecon_H");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconOp<double, 2>>("D2_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_D2_D_veq_sprecon_pH(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_D2_D_veq_sprecon_pH");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconOp<double, 2>>("D2_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_D2_D_vpeq_sprecon_H(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_D2_D_vpeq_sprecon_H");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconOp<double, 2>>("D2_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_D2_D_vpeq_sprecon_pH(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_D2_D_vpeq_sprecon_pH");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconOp<double, 2>>("D2_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_D2_D_vmeq_sprecon_H(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_D2_D_vmeq_sprecon_H");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconOp<double, 2>>("D2_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_D2_D_vmeq_sprecon_pH(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_D2_D_vmeq_sprecon_pH");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconOp<double, 2>>("D2_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_D2_D_veqm_sprecon_H(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_D2_D_veqm_sprecon_H");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconOp<double, 2>>("D2_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_D2_D_veqm_sprecon_pH(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_D2_D_veqm_sprecon_pH");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconOp<double, 2>>("D2_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_D2_D_xeq_sprecon_H(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_sprecon_H");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconOp<double, 2>>("D2_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_D2_D_xeq_sprecon_pH(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_sprecon_pH");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconOp<double, 2>>("D2_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_D2_D_xpeq_sprecon_H(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xpeq_sprecon_H");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconOp<double, 2>>("D2_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_D2_D_xpeq_sprecon_pH(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xpeq_sprecon_pH");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconOp<double, 2>>("D2_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_D2_D_xmeq_sprecon_H(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xmeq_sprecon_H");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconOp<double, 2>>("D2_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_D2_D_xmeq_sprecon_pH(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xmeq_sprecon_pH");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconOp<double, 2>>("D2_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_D2_D_xeqm_sprecon_H(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeqm_sprecon_H");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconOp<double, 2>>("D2_sprecon", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_D2_D_xeqm_sprecon_pH(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeqm_sprecon_pH");
  if (mu < 0 || mu > 4) return;
  qlab::api_map<qlab::SpreconOp<double, 2>>("D2_sprecon", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign);
}

}  // extern "C"
