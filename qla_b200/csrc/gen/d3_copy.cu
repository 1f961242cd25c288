// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA D3 copy entry points (extern "C"), reference: lib/perl/build_qla.pl:370-400 (assignment / gather)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"

extern "C" {
QLAB_EXPORT void QLA_D3_V_veq_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D3_V_veq_V");
  qlab::api_map<qlab::CopyOp<double, 3>>("D3_copy_V", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_V_veq_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D3_V_veq_pV");
  qlab::api_map<qlab::CopyOp<double, 3>>("D3_copy_V", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_V_vpeq_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D3_V_vpeq_V");
  qlab::api_map<qlab::CopyOp<double, 3>>("D3_copy_V", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_V_vpeq_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D3_V_vpeq_pV");
  qlab::api_map<qlab::CopyOp<double, 3>>("D3_copy_V", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_V_vmeq_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D3_V_vmeq_V");
  qlab::api_map<qlab::CopyOp<double, 3>>("D3_copy_V", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_V_vmeq_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D3_V_vmeq_pV");
  qlab::api_map<qlab::CopyOp<double, 3>>("D3_copy_V", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_V_veqm_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D3_V_veqm_V");
  qlab::api_map<qlab::CopyOp<double, 3>>("D3_copy_V", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_V_veqm_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D3_V_veqm_pV");
  qlab::api_map<qlab::CopyOp<double, 3>>("D3_copy_V", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_V_xeq_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xeq_V");
  qlab::api_map<qlab::CopyOp<double, 3>>("D3_copy_V", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_V_xeq_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xeq_pV");
  qlab::api_map<qlab::CopyOp<double, 3>>("D3_copy_V", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_V_xpeq_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xpeq_V");
  qlab::api_map<qlab::CopyOp<double, 3>>("D3_copy_V", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_V_xpeq_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xpeq_pV");
  qlab::api_map<qlab::CopyOp<double, 3>>("D3_copy_V", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_V_xmeq_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xmeq_V");
  qlab::api_map<qlab::CopyOp<double, 3>>("D3_copy_V", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_V_xmeq_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xmeq_pV");
  qlab::api_map<qlab::CopyOp<double, 3>>("D3_copy_V", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_V_xeqm_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xeqm_V");
  qlab::api_map<qlab::CopyOp<double, 3>>("D3_copy_V", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_V_xeqm_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xeqm_pV");
  qlab::api_map<qlab::CopyOp<double, 3>>("D3_copy_V", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_V_eq_xV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ a, int * ja, int n) {
  QLAB_TRACE("QLA_D3_V_eq_xV");
  qlab::api_map<qlab::CopyOp<double, 3>>("D3_copy_V", r, qlab::op_idx(a, ja), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_V_peq_xV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ a, int * ja, int n) {
  QLAB_TRACE("QLA_D3_V_peq_xV");
  qlab::api_map<qlab::CopyOp<double, 3>>("D3_copy_V", r, qlab::op_idx(a, ja), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_V_meq_xV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ a, int * ja, int n) {
  QLAB_TRACE("QLA_D3_V_meq_xV");
  qlab::api_map<qlab::CopyOp<double, 3>>("D3_copy_V", r, qlab::op_idx(a, ja), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_V_eqm_xV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorVector *__restrict__ a, int * ja, int n) {
  QLAB_TRACE("QLA_D3_V_eqm_xV");
  qlab::api_map<qlab::CopyOp<double, 3>>("D3_copy_V", r, qlab::op_idx(a, ja), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_H_veq_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D3_H_veq_H");
  qlab::api_map<qlab::CopyOp<double, 6>>("D3_copy_H", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_H_veq_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D3_H_veq_pH");
  qlab::api_map<qlab::CopyOp<double, 6>>("D3_copy_H", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_H_vpeq_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D3_H_vpeq_H");
  qlab::api_map<qlab::CopyOp<double, 6>>("D3_copy_H", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_H_vpeq_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D3_H_vpeq_pH");
  qlab::api_map<qlab::CopyOp<double, 6>>("D3_copy_H", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_H_vmeq_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D3_H_vmeq_H");
  qlab::api_map<qlab::CopyOp<double, 6>>("D3_copy_H", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_H_vmeq_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D3_H_vmeq_pH");
  qlab::api_map<qlab::CopyOp<double, 6>>("D3_copy_H", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_H_veqm_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D3_H_veqm_H");
  qlab::api_map<qlab::CopyOp<double, 6>>("D3_copy_H", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_H_veqm_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D3_H_veqm_pH");
  qlab::api_map<qlab::CopyOp<double, 6>>("D3_copy_H", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_H_xeq_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xeq_H");
  qlab::api_map<qlab::CopyOp<double, 6>>("D3_copy_H", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_H_xeq_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xeq_pH");
  qlab::api_map<qlab::CopyOp<double, 6>>("D3_copy_H", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_H_xpeq_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xpeq_H");
  qlab::api_map<qlab::CopyOp<double, 6>>("D3_copy_H", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_H_xpeq_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xpeq_pH");
  qlab::api_map<qlab::CopyOp<double, 6>>("D3_copy_H", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_H_xmeq_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xmeq_H");
  qlab::api_map<qlab::CopyOp<double, 6>>("D3_copy_H", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_H_xmeq_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xmeq_pH");
  qlab::api_map<qlab::CopyOp<double, 6>>("D3_copy_H", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_H_xeqm_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xeqm_H");
  qlab::api_map<qlab::CopyOp<double, 6>>("D3_copy_H", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_H_xeqm_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xeqm_pH");
  qlab::api_map<qlab::CopyOp<double, 6>>("D3_copy_H", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_H_eq_xH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ a, int * ja, int n) {
  QLAB_TRACE("QLA_D3_H_eq_xH");
  qlab::api_map<qlab::CopyOp<double, 6>>("D3_copy_H", r, qlab::op_idx(a, ja), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_H_peq_xH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ a, int * ja, int n) {
  QLAB_TRACE("QLA_D3_H_peq_xH");
  qlab::api_map<qlab::CopyOp<double, 6>>("D3_copy_H", r, qlab::op_idx(a, ja), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_H_meq_xH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ a, int * ja, int n) {
  QLAB_TRACE("QLA_D3_H_meq_xH");
  qlab::api_map<qlab::CopyOp<double, 6>>("D3_copy_H", r, qlab::op_idx(a, ja), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_H_eqm_xH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_HalfFermion *__restrict__ a, int * ja, int n) {
  QLAB_TRACE("QLA_D3_H_eqm_xH");
  qlab::api_map<qlab::CopyOp<double, 6>>("D3_copy_H", r, qlab::op_idx(a, ja), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_D_veq_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D3_D_veq_D");
  qlab::api_map<qlab::CopyOp<double, 12>>("D3_copy_D", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_D_veq_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D3_D_veq_pD");
  qlab::api_map<qlab::CopyOp<double, 12>>("D3_copy_D", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_D_vpeq_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D3_D_vpeq_D");
  qlab::api_map<qlab::CopyOp<double, 12>>("D3_copy_D", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_D_vpeq_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D3_D_vpeq_pD");
  qlab::api_map<qlab::CopyOp<double, 12>>("D3_copy_D", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_D_vmeq_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D3_D_vmeq_D");
  qlab::api_map<qlab::CopyOp<double, 12>>("D3_copy_D", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_D_vmeq_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D3_D_vmeq_pD");
  qlab::api_map<qlab::CopyOp<double, 12>>("D3_copy_D", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_D_veqm_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D3_D_veqm_D");
  qlab::api_map<qlab::CopyOp<double, 12>>("D3_copy_D", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_D_veqm_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D3_D_veqm_pD");
  qlab::api_map<qlab::CopyOp<double, 12>>("D3_copy_D", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_D_xeq_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xeq_D");
  qlab::api_map<qlab::CopyOp<double, 12>>("D3_copy_D", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_D_xeq_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xeq_pD");
  qlab::api_map<qlab::CopyOp<double, 12>>("D3_copy_D", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_D_xpeq_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xpeq_D");
  qlab::api_map<qlab::CopyOp<double, 12>>("D3_copy_D", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_D_xpeq_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xpeq_pD");
  qlab::api_map<qlab::CopyOp<double, 12>>("D3_copy_D", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_D_xmeq_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xmeq_D");
  qlab::api_map<qlab::CopyOp<double, 12>>("D3_copy_D", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_D_xmeq_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xmeq_pD");
  qlab::api_map<qlab::CopyOp<double, 12>>("D3_copy_D", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_D_xeqm_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xeqm_D");
  qlab::api_map<qlab::CopyOp<double, 12>>("D3_copy_D", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_D_xeqm_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xeqm_pD");
  qlab::api_map<qlab::CopyOp<double, 12>>("D3_copy_D", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_D_eq_xD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ a, int * ja, int n) {
  QLAB_TRACE("QLA_D3_D_eq_xD");
  qlab::api_map<qlab::CopyOp<double, 12>>("D3_copy_D", r, qlab::op_idx(a, ja), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_D_peq_xD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ a, int * ja, int n) {
  QLAB_TRACE("QLA_D3_D_peq_xD");
  qlab::api_map<qlab::CopyOp<double, 12>>("D3_copy_D", r, qlab::op_idx(a, ja), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_D_meq_xD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ a, int * ja, int n) {
  QLAB_TRACE("QLA_D3_D_meq_xD");
  qlab::api_map<qlab::CopyOp<double, 12>>("D3_copy_D", r, qlab::op_idx(a, ja), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_D_eqm_xD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_DiracFermion *__restrict__ a, int * ja, int n) {
  QLAB_TRACE("QLA_D3_D_eqm_xD");
  qlab::api_map<qlab::CopyOp<double, 12>>("D3_copy_D", r, qlab::op_idx(a, ja), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_veq_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D3_M_veq_M");
  qlab::api_map<qlab::CopyOp<double, 9>>("D3_copy_M", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_veq_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D3_M_veq_pM");
  qlab::api_map<qlab::CopyOp<double, 9>>("D3_copy_M", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_vpeq_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D3_M_vpeq_M");
  qlab::api_map<qlab::CopyOp<double, 9>>("D3_copy_M", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_vpeq_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D3_M_vpeq_pM");
  qlab::api_map<qlab::CopyOp<double, 9>>("D3_copy_M", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_vmeq_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D3_M_vmeq_M");
  qlab::api_map<qlab::CopyOp<double, 9>>("D3_copy_M", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_vmeq_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D3_M_vmeq_pM");
  qlab::api_map<qlab::CopyOp<double, 9>>("D3_copy_M", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_veqm_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D3_M_veqm_M");
  qlab::api_map<qlab::CopyOp<double, 9>>("D3_copy_M", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_veqm_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D3_M_veqm_pM");
  qlab::api_map<qlab::CopyOp<double, 9>>("D3_copy_M", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_xeq_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeq_M");
  qlab::api_map<qlab::CopyOp<double, 9>>("D3_copy_M", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_xeq_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeq_pM");
  qlab::api_map<qlab::CopyOp<double, 9>>("D3_copy_M", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_xpeq_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xpeq_M");
  qlab::api_map<qlab::CopyOp<double, 9>>("D3_copy_M", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_xpeq_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xpeq_pM");
  qlab::api_map<qlab::CopyOp<double, 9>>("D3_copy_M", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_xmeq_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xmeq_M");
  qlab::api_map<qlab::CopyOp<double, 9>>("D3_copy_M", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_xmeq_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xmeq_pM");
  qlab::api_map<qlab::CopyOp<double, 9>>("D3_copy_M", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_xeqm_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeqm_M");
  qlab::api_map<qlab::CopyOp<double, 9>>("D3_copy_M", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_xeqm_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeqm_pM");
  qlab::api_map<qlab::CopyOp<double, 9>>("D3_copy_M", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_eq_xM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, int * ja, int n) {
  QLAB_TRACE("QLA_D3_M_eq_xM");
  qlab::api_map<qlab::CopyOp<double, 9>>("D3_copy_M", r, qlab::op_idx(a, ja), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_peq_xM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, int * ja, int n) {
  QLAB_TRACE("QLA_D3_M_peq_xM");
  qlab::api_map<qlab::CopyOp<double, 9>>("D3_copy_M", r, qlab::op_idx(a, ja), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_meq_xM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, int * ja, int n) {
  QLAB_TRACE("QLA_D3_M_meq_xM");
  qlab::api_map<qlab::CopyOp<double, 9>>("D3_copy_M", r, qlab::op_idx(a, ja), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_eqm_xM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, int * ja, int n) {
  QLAB_TRACE("QLA_D3_M_eqm_xM");
  qlab::api_map<qlab::CopyOp<double, 9>>("D3_copy_M", r, qlab::op_idx(a, ja), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

}  // extern "C"
