// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F3 spproj entry points (extern "C"), reference: lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"

extern "C" {
QLAB_EXPORT void QLA_F3_H_veq_spproj_D(QLA_F3_HalfFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F3_H_veq_spproj_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojOp<float, 3>>("F3_spproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F3_H_veq_spproj_pD(QLA_F3_HalfFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F3_H_veq_spproj_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojOp<float, 3>>("F3_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F3_H_vpeq_spproj_D(QLA_F3_HalfFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F3_H_vpeq_spproj_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojOp<float, 3>>("F3_spproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F3_H_vpeq_spproj_pD(QLA_F3_HalfFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F3_H_vpeq_spproj_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojOp<float, 3>>("F3_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F3_H_vmeq_spproj_D(QLA_F3_HalfFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F3_H_vmeq_spproj_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojOp<float, 3>>("F3_spproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F3_H_vmeq_spproj_pD(QLA_F3_HalfFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F3_H_vmeq_spproj_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojOp<float, 3>>("F3_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F3_H_veqm_spproj_D(QLA_F3_HalfFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F3_H_veqm_spproj_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojOp<float, 3>>("F3_spproj", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F3_H_veqm_spproj_pD(QLA_F3_HalfFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int mu, int sign, int n) {
  QLAB_TRACE("QLA_F3_H_veqm_spproj_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojOp<float, 3>>("F3_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F3_H_xeq_spproj_D(QLA_F3_HalfFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F3_H_xeq_spproj_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojOp<float, 3>>("F3_spproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F3_H_xeq_spproj_pD(QLA_F3_HalfFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F3_H_xeq_spproj_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojOp<float, 3>>("F3_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ, mu, sign);
}

QLAB_EXPORT void QLA_F3_H_xpeq_spproj_D(QLA_F3_HalfFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F3_H_xpeq_spproj_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojOp<float, 3>>("F3_spproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F3_H_xpeq_spproj_pD(QLA_F3_HalfFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F3_H_xpeq_spproj_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojOp<float, 3>>("F3_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ, mu, sign);
}

QLAB_EXPORT void QLA_F3_H_xmeq_spproj_D(QLA_F3_HalfFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F3_H_xmeq_spproj_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojOp<float, 3>>("F3_spproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F3_H_xmeq_spproj_pD(QLA_F3_HalfFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F3_H_xmeq_spproj_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojOp<float, 3>>("F3_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ, mu, sign);
}

QLAB_EXPORT void QLA_F3_H_xeqm_spproj_D(QLA_F3_HalfFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F3_H_xeqm_spproj_D");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojOp<float, 3>>("F3_spproj", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign);
}

QLAB_EXPORT void QLA_F3_H_xeqm_spproj_pD(QLA_F3_HalfFermion *__restrict__ r, QLA_F3_DiracFermion *__restrict__ * a, int mu, int sign, int * index, int n) {
  QLAB_TRACE("QLA_F3_H_xeqm_spproj_pD");
  if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */
  qlab::api_map<qlab::SpprojOp<float, 3>>("F3_spproj", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM, mu, sign);
}

}  // extern "C"
