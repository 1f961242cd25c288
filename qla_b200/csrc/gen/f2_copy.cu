// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F2 copy entry points (extern "C"), reference: lib/perl/build_qla.pl:370-400 (assignment / gather)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"

extern "C" {
QLAB_EXPORT void QLA_F2_V_veq_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_V_veq_V");
  qlab::api_map<qlab::CopyOp<float, 2>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_veq_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_V_veq_pV");
  qlab::api_map<qlab::CopyOp<float, 2>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_V_vpeq_V");
  qlab::api_map<qlab::CopyOp<float, 2>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vpeq_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_V_vpeq_pV");
  qlab::api_map<qlab::CopyOp<float, 2>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_V_vmeq_V");
  qlab::api_map<qlab::CopyOp<float, 2>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_vmeq_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_V_vmeq_pV");
  qlab::api_map<qlab::CopyOp<float, 2>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_veqm_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_V_veqm_V");
  qlab::api_map<qlab::CopyOp<float, 2>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_veqm_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_V_veqm_pV");
  qlab::api_map<qlab::CopyOp<float, 2>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeq_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_V");
  qlab::api_map<qlab::CopyOp<float, 2>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xeq_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeq_pV");
  qlab::api_map<qlab::CopyOp<float, 2>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xpeq_V");
  qlab::api_map<qlab::CopyOp<float, 2>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xpeq_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xpeq_pV");
  qlab::api_map<qlab::CopyOp<float, 2>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xmeq_V");
  qlab::api_map<qlab::CopyOp<float, 2>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xmeq_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xmeq_pV");
  qlab::api_map<qlab::CopyOp<float, 2>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_V_xeqm_V(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeqm_V");
  qlab::api_map<qlab::CopyOp<float, 2>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_V_xeqm_pV(QLA_F2_ColorVector *__restrict__ r, QLA_F2_ColorVector *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_V_xeqm_pV");
  qlab::api_map<qlab::CopyOp<float, 2>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_H_veq_H(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_H_veq_H");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_H_veq_pH(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_H_veq_pH");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_H_vpeq_H(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_H_vpeq_H");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_H_vpeq_pH(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_H_vpeq_pH");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_H_vmeq_H(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_H_vmeq_H");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_H_vmeq_pH(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_H_vmeq_pH");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_H_veqm_H(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_H_veqm_H");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_H_veqm_pH(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_H_veqm_pH");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_H_xeq_H(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeq_H");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_H_xeq_pH(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeq_pH");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_H_xpeq_H(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xpeq_H");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_H_xpeq_pH(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xpeq_pH");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_H_xmeq_H(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xmeq_H");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_H_xmeq_pH(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xmeq_pH");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_H_xeqm_H(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeqm_H");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_H_xeqm_pH(QLA_F2_HalfFermion *__restrict__ r, QLA_F2_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_H_xeqm_pH");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_D_veq_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_D_veq_D");
  qlab::api_map<qlab::CopyOp<float, 8>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_D_veq_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_D_veq_pD");
  qlab::api_map<qlab::CopyOp<float, 8>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_D_vpeq_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_D_vpeq_D");
  qlab::api_map<qlab::CopyOp<float, 8>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_D_vpeq_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_D_vpeq_pD");
  qlab::api_map<qlab::CopyOp<float, 8>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_D_vmeq_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_D_vmeq_D");
  qlab::api_map<qlab::CopyOp<float, 8>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_D_vmeq_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_D_vmeq_pD");
  qlab::api_map<qlab::CopyOp<float, 8>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_D_veqm_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_D_veqm_D");
  qlab::api_map<qlab::CopyOp<float, 8>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_D_veqm_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_D_veqm_pD");
  qlab::api_map<qlab::CopyOp<float, 8>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_D_xeq_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_D");
  qlab::api_map<qlab::CopyOp<float, 8>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_D_xeq_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeq_pD");
  qlab::api_map<qlab::CopyOp<float, 8>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_D_xpeq_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xpeq_D");
  qlab::api_map<qlab::CopyOp<float, 8>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_D_xpeq_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xpeq_pD");
  qlab::api_map<qlab::CopyOp<float, 8>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_D_xmeq_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xmeq_D");
  qlab::api_map<qlab::CopyOp<float, 8>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_D_xmeq_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xmeq_pD");
  qlab::api_map<qlab::CopyOp<float, 8>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_D_xeqm_D(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeqm_D");
  qlab::api_map<qlab::CopyOp<float, 8>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_D_xeqm_pD(QLA_F2_DiracFermion *__restrict__ r, QLA_F2_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_D_xeqm_pD");
  qlab::api_map<qlab::CopyOp<float, 8>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_M_veq_M(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_M_veq_M");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_M_veq_pM(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_M_veq_pM");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_M_vpeq_M(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_M_vpeq_M");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_M_vpeq_pM(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_M_vpeq_pM");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_M_vmeq_M(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_M_vmeq_M");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_M_vmeq_pM(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_M_vmeq_pM");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_M_veqm_M(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F2_M_veqm_M");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_M_veqm_pM(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F2_M_veqm_pM");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_M_xeq_M(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xeq_M");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_M_xeq_pM(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xeq_pM");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F2_M_xpeq_M(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xpeq_M");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_M_xpeq_pM(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xpeq_pM");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F2_M_xmeq_M(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xmeq_M");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_M_xmeq_pM(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xmeq_pM");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F2_M_xeqm_M(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xeqm_M");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F2_M_xeqm_pM(QLA_F2_ColorMatrix *__restrict__ r, QLA_F2_ColorMatrix *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F2_M_xeqm_pM");
  qlab::api_map<qlab::CopyOp<float, 4>>("F2_copy", r, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

}  // extern "C"
