// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA D3 lmult entry points (extern "C"), reference: lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), expressions_tensor.pl:766
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"

extern "C" {
QLAB_EXPORT void QLA_D3_V_veq_M_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_V_veq_M_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_V_veq_M_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_V_veq_M_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_V_veq_Ma_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_V_veq_Ma_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_V_veq_Ma_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_V_veq_Ma_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_V_veq_pM_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_V_veq_pM_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_V_veq_pM_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_V_veq_pM_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_V_veq_pMa_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_V_veq_pMa_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_V_veq_pMa_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_V_veq_pMa_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_V_vpeq_M_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_V_vpeq_M_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_V_vpeq_M_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_V_vpeq_M_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_V_vpeq_Ma_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_V_vpeq_Ma_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_V_vpeq_Ma_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_V_vpeq_Ma_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_V_vpeq_pM_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_V_vpeq_pM_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_V_vpeq_pM_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_V_vpeq_pM_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_V_vpeq_pMa_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_V_vpeq_pMa_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_V_vpeq_pMa_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_V_vpeq_pMa_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_V_vmeq_M_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_V_vmeq_M_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_V_vmeq_M_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_V_vmeq_M_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_V_vmeq_Ma_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_V_vmeq_Ma_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_V_vmeq_Ma_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_V_vmeq_Ma_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_V_vmeq_pM_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_V_vmeq_pM_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_V_vmeq_pM_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_V_vmeq_pM_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_V_vmeq_pMa_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_V_vmeq_pMa_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_V_vmeq_pMa_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_V_vmeq_pMa_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_V_veqm_M_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_V_veqm_M_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_V_veqm_M_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_V_veqm_M_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_V_veqm_Ma_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_V_veqm_Ma_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_V_veqm_Ma_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_V_veqm_Ma_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_V_veqm_pM_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_V_veqm_pM_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_V_veqm_pM_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_V_veqm_pM_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_V_veqm_pMa_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_V_veqm_pMa_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_V_veqm_pMa_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_V_veqm_pMa_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_V_xeq_M_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xeq_M_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_V_xeq_M_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xeq_M_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_V_xeq_Ma_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xeq_Ma_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_V_xeq_Ma_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xeq_Ma_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_V_xeq_pM_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xeq_pM_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_V_xeq_pM_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xeq_pM_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_V_xeq_pMa_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xeq_pMa_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_V_xeq_pMa_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xeq_pMa_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_V_xpeq_M_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xpeq_M_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_V_xpeq_M_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xpeq_M_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_V_xpeq_Ma_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xpeq_Ma_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_V_xpeq_Ma_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xpeq_Ma_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_V_xpeq_pM_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xpeq_pM_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_V_xpeq_pM_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xpeq_pM_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_V_xpeq_pMa_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xpeq_pMa_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_V_xpeq_pMa_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xpeq_pMa_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_V_xmeq_M_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xmeq_M_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_V_xmeq_M_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xmeq_M_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_V_xmeq_Ma_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xmeq_Ma_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_V_xmeq_Ma_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xmeq_Ma_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_V_xmeq_pM_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xmeq_pM_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_V_xmeq_pM_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xmeq_pM_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_V_xmeq_pMa_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xmeq_pMa_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_V_xmeq_pMa_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xmeq_pMa_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_V_xeqm_M_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xeqm_M_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_V_xeqm_M_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xeqm_M_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_V_xeqm_Ma_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xeqm_Ma_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_V_xeqm_Ma_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xeqm_Ma_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_V_xeqm_pM_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xeqm_pM_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_V_xeqm_pM_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xeqm_pM_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_V_xeqm_pMa_times_V(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xeqm_pMa_times_V");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_V_xeqm_pMa_times_pV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorVector *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_V_xeqm_pMa_times_pV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_V_eq_M_times_xV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_V_eq_M_times_xV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_V_eq_Ma_times_xV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_V_eq_Ma_times_xV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_V_peq_M_times_xV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_V_peq_M_times_xV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_V_peq_Ma_times_xV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_V_peq_Ma_times_xV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_V_meq_M_times_xV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_V_meq_M_times_xV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_V_meq_Ma_times_xV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_V_meq_Ma_times_xV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_V_eqm_M_times_xV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_V_eqm_M_times_xV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, false, false>>("D3_lmult_V00", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_V_eqm_Ma_times_xV(QLA_D3_ColorVector *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorVector *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_V_eqm_Ma_times_xV");
  qlab::api_map<qlab::LMultOp<double, 3, 1, true, false>>("D3_lmult_V10", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_H_veq_M_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_H_veq_M_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_H_veq_M_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_H_veq_M_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_H_veq_Ma_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_H_veq_Ma_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_H_veq_Ma_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_H_veq_Ma_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_H_veq_pM_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_H_veq_pM_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_H_veq_pM_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_H_veq_pM_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_H_veq_pMa_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_H_veq_pMa_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_H_veq_pMa_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_H_veq_pMa_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_H_vpeq_M_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_H_vpeq_M_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_H_vpeq_M_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_H_vpeq_M_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_H_vpeq_Ma_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_H_vpeq_Ma_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_H_vpeq_Ma_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_H_vpeq_Ma_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_H_vpeq_pM_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_H_vpeq_pM_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_H_vpeq_pM_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_H_vpeq_pM_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_H_vpeq_pMa_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_H_vpeq_pMa_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_H_vpeq_pMa_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_H_vpeq_pMa_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_H_vmeq_M_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_H_vmeq_M_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_H_vmeq_M_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_H_vmeq_M_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_H_vmeq_Ma_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_H_vmeq_Ma_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_H_vmeq_Ma_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_H_vmeq_Ma_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_H_vmeq_pM_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_H_vmeq_pM_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_H_vmeq_pM_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_H_vmeq_pM_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_H_vmeq_pMa_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_H_vmeq_pMa_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_H_vmeq_pMa_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_H_vmeq_pMa_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_H_veqm_M_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_H_veqm_M_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_H_veqm_M_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_H_veqm_M_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_H_veqm_Ma_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_H_veqm_Ma_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_H_veqm_Ma_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_H_veqm_Ma_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_H_veqm_pM_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_H_veqm_pM_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_H_veqm_pM_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_H_veqm_pM_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_H_veqm_pMa_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_H_veqm_pMa_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_H_veqm_pMa_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_H_veqm_pMa_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_H_xeq_M_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xeq_M_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_H_xeq_M_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xeq_M_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_H_xeq_Ma_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xeq_Ma_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_H_xeq_Ma_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xeq_Ma_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_H_xeq_pM_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xeq_pM_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_H_xeq_pM_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xeq_pM_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_H_xeq_pMa_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xeq_pMa_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_H_xeq_pMa_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xeq_pMa_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_H_xpeq_M_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xpeq_M_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_H_xpeq_M_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xpeq_M_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_H_xpeq_Ma_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xpeq_Ma_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_H_xpeq_Ma_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xpeq_Ma_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_H_xpeq_pM_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xpeq_pM_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_H_xpeq_pM_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xpeq_pM_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_H_xpeq_pMa_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xpeq_pMa_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_H_xpeq_pMa_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xpeq_pMa_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_H_xmeq_M_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xmeq_M_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_H_xmeq_M_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xmeq_M_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_H_xmeq_Ma_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xmeq_Ma_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_H_xmeq_Ma_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xmeq_Ma_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_H_xmeq_pM_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xmeq_pM_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_H_xmeq_pM_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xmeq_pM_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_H_xmeq_pMa_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xmeq_pMa_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_H_xmeq_pMa_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xmeq_pMa_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_H_xeqm_M_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xeqm_M_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_H_xeqm_M_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xeqm_M_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_H_xeqm_Ma_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xeqm_Ma_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_H_xeqm_Ma_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xeqm_Ma_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_H_xeqm_pM_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xeqm_pM_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_H_xeqm_pM_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xeqm_pM_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_H_xeqm_pMa_times_H(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xeqm_pMa_times_H");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_H_xeqm_pMa_times_pH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_H_xeqm_pMa_times_pH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_H_eq_M_times_xH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_H_eq_M_times_xH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_H_eq_Ma_times_xH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_H_eq_Ma_times_xH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_H_peq_M_times_xH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_H_peq_M_times_xH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_H_peq_Ma_times_xH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_H_peq_Ma_times_xH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_H_meq_M_times_xH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_H_meq_M_times_xH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_H_meq_Ma_times_xH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_H_meq_Ma_times_xH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_H_eqm_M_times_xH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_H_eqm_M_times_xH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, false, false>>("D3_lmult_H00", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_H_eqm_Ma_times_xH(QLA_D3_HalfFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_HalfFermion *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_H_eqm_Ma_times_xH");
  qlab::api_map<qlab::LMultOp<double, 3, 2, true, false>>("D3_lmult_H10", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_D_veq_M_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_D_veq_M_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_D_veq_M_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_D_veq_M_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_D_veq_Ma_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_D_veq_Ma_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_D_veq_Ma_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_D_veq_Ma_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_D_veq_pM_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_D_veq_pM_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_D_veq_pM_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_D_veq_pM_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_D_veq_pMa_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_D_veq_pMa_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_D_veq_pMa_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_D_veq_pMa_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_D_vpeq_M_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_D_vpeq_M_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_D_vpeq_M_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_D_vpeq_M_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_D_vpeq_Ma_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_D_vpeq_Ma_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_D_vpeq_Ma_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_D_vpeq_Ma_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_D_vpeq_pM_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_D_vpeq_pM_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_D_vpeq_pM_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_D_vpeq_pM_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_D_vpeq_pMa_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_D_vpeq_pMa_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_D_vpeq_pMa_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_D_vpeq_pMa_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_D_vmeq_M_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_D_vmeq_M_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_D_vmeq_M_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_D_vmeq_M_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_D_vmeq_Ma_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_D_vmeq_Ma_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_D_vmeq_Ma_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_D_vmeq_Ma_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_D_vmeq_pM_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_D_vmeq_pM_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_D_vmeq_pM_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_D_vmeq_pM_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_D_vmeq_pMa_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_D_vmeq_pMa_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_D_vmeq_pMa_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_D_vmeq_pMa_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_D_veqm_M_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_D_veqm_M_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_D_veqm_M_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_D_veqm_M_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_D_veqm_Ma_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_D_veqm_Ma_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_D_veqm_Ma_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_D_veqm_Ma_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_D_veqm_pM_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_D_veqm_pM_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_D_veqm_pM_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_D_veqm_pM_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_D_veqm_pMa_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_D_veqm_pMa_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_D_veqm_pMa_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_D_veqm_pMa_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_D_xeq_M_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xeq_M_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_D_xeq_M_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xeq_M_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_D_xeq_Ma_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xeq_Ma_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_D_xeq_Ma_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xeq_Ma_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_D_xeq_pM_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xeq_pM_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_D_xeq_pM_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xeq_pM_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_D_xeq_pMa_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xeq_pMa_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_D_xeq_pMa_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xeq_pMa_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_D_xpeq_M_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xpeq_M_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_D_xpeq_M_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xpeq_M_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_D_xpeq_Ma_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xpeq_Ma_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_D_xpeq_Ma_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xpeq_Ma_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_D_xpeq_pM_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xpeq_pM_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_D_xpeq_pM_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xpeq_pM_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_D_xpeq_pMa_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xpeq_pMa_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_D_xpeq_pMa_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xpeq_pMa_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_D_xmeq_M_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xmeq_M_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_D_xmeq_M_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xmeq_M_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_D_xmeq_Ma_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xmeq_Ma_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_D_xmeq_Ma_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xmeq_Ma_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_D_xmeq_pM_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xmeq_pM_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_D_xmeq_pM_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xmeq_pM_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_D_xmeq_pMa_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xmeq_pMa_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_D_xmeq_pMa_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xmeq_pMa_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_D_xeqm_M_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xeqm_M_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_D_xeqm_M_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xeqm_M_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_D_xeqm_Ma_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xeqm_Ma_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_D_xeqm_Ma_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xeqm_Ma_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_D_xeqm_pM_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xeqm_pM_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_D_xeqm_pM_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xeqm_pM_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_D_xeqm_pMa_times_D(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xeqm_pMa_times_D");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_D_xeqm_pMa_times_pD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_D_xeqm_pMa_times_pD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_D_eq_M_times_xD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_D_eq_M_times_xD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_D_eq_Ma_times_xD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_D_eq_Ma_times_xD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_D_peq_M_times_xD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_D_peq_M_times_xD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_D_peq_Ma_times_xD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_D_peq_Ma_times_xD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_D_meq_M_times_xD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_D_meq_M_times_xD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_D_meq_Ma_times_xD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_D_meq_Ma_times_xD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_D_eqm_M_times_xD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_D_eqm_M_times_xD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, false, false>>("D3_lmult_D00", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_D_eqm_Ma_times_xD(QLA_D3_DiracFermion *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_DiracFermion *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_D_eqm_Ma_times_xD");
  qlab::api_map<qlab::LMultOp<double, 3, 4, true, false>>("D3_lmult_D10", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_veq_M_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_veq_M_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_veq_M_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_veq_M_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_veq_M_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_veq_M_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_veq_M_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_veq_M_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_veq_Ma_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_veq_Ma_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_veq_Ma_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_veq_Ma_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_veq_Ma_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_veq_Ma_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_veq_Ma_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_veq_Ma_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_veq_pM_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_veq_pM_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_veq_pM_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_veq_pM_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_veq_pM_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_veq_pM_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_veq_pM_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_veq_pM_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_veq_pMa_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_veq_pMa_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_veq_pMa_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_veq_pMa_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_veq_pMa_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_veq_pMa_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_veq_pMa_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_veq_pMa_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_vpeq_M_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_vpeq_M_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_vpeq_M_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_vpeq_M_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_vpeq_M_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_vpeq_M_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_vpeq_M_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_vpeq_M_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_vpeq_Ma_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_vpeq_Ma_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_vpeq_Ma_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_vpeq_Ma_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_vpeq_Ma_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_vpeq_Ma_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_vpeq_Ma_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_vpeq_Ma_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_vpeq_pM_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_vpeq_pM_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_vpeq_pM_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_vpeq_pM_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_vpeq_pM_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_vpeq_pM_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_vpeq_pM_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_vpeq_pM_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_vpeq_pMa_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_vpeq_pMa_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_vpeq_pMa_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_vpeq_pMa_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_vpeq_pMa_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_vpeq_pMa_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_vpeq_pMa_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_vpeq_pMa_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_vmeq_M_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_vmeq_M_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_vmeq_M_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_vmeq_M_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_vmeq_M_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_vmeq_M_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_vmeq_M_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_vmeq_M_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_vmeq_Ma_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_vmeq_Ma_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_vmeq_Ma_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_vmeq_Ma_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_vmeq_Ma_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_vmeq_Ma_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_vmeq_Ma_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_vmeq_Ma_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_vmeq_pM_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_vmeq_pM_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_vmeq_pM_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_vmeq_pM_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_vmeq_pM_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_vmeq_pM_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_vmeq_pM_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_vmeq_pM_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_vmeq_pMa_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_vmeq_pMa_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_vmeq_pMa_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_vmeq_pMa_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_vmeq_pMa_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_vmeq_pMa_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_vmeq_pMa_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_vmeq_pMa_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_veqm_M_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_veqm_M_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_veqm_M_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_veqm_M_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_veqm_M_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_veqm_M_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_veqm_M_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_veqm_M_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_veqm_Ma_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_veqm_Ma_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_veqm_Ma_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_veqm_Ma_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_veqm_Ma_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_veqm_Ma_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_veqm_Ma_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_veqm_Ma_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_veqm_pM_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_veqm_pM_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_veqm_pM_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_veqm_pM_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_veqm_pM_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_veqm_pM_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_veqm_pM_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_veqm_pM_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_veqm_pMa_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_veqm_pMa_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_veqm_pMa_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_veqm_pMa_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_veqm_pMa_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D3_M_veqm_pMa_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_veqm_pMa_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D3_M_veqm_pMa_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_xeq_M_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeq_M_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_xeq_M_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeq_M_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_xeq_M_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeq_M_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_xeq_M_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeq_M_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_xeq_Ma_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeq_Ma_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_xeq_Ma_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeq_Ma_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_xeq_Ma_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeq_Ma_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_xeq_Ma_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeq_Ma_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_xeq_pM_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeq_pM_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_xeq_pM_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeq_pM_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_xeq_pM_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeq_pM_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_xeq_pM_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeq_pM_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_xeq_pMa_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeq_pMa_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_xeq_pMa_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeq_pMa_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_xeq_pMa_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeq_pMa_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_xeq_pMa_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeq_pMa_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_xpeq_M_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xpeq_M_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_xpeq_M_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xpeq_M_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_xpeq_M_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xpeq_M_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_xpeq_M_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xpeq_M_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_xpeq_Ma_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xpeq_Ma_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_xpeq_Ma_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xpeq_Ma_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_xpeq_Ma_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xpeq_Ma_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_xpeq_Ma_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xpeq_Ma_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_xpeq_pM_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xpeq_pM_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_xpeq_pM_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xpeq_pM_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_xpeq_pM_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xpeq_pM_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_xpeq_pM_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xpeq_pM_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_xpeq_pMa_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xpeq_pMa_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_xpeq_pMa_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xpeq_pMa_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_xpeq_pMa_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xpeq_pMa_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_xpeq_pMa_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xpeq_pMa_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_xmeq_M_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xmeq_M_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_xmeq_M_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xmeq_M_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_xmeq_M_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xmeq_M_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_xmeq_M_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xmeq_M_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_xmeq_Ma_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xmeq_Ma_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_xmeq_Ma_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xmeq_Ma_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_xmeq_Ma_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xmeq_Ma_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_xmeq_Ma_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xmeq_Ma_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_xmeq_pM_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xmeq_pM_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_xmeq_pM_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xmeq_pM_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_xmeq_pM_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xmeq_pM_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_xmeq_pM_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xmeq_pM_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_xmeq_pMa_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xmeq_pMa_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_xmeq_pMa_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xmeq_pMa_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_xmeq_pMa_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xmeq_pMa_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_xmeq_pMa_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xmeq_pMa_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_xeqm_M_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeqm_M_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_xeqm_M_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeqm_M_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_xeqm_M_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeqm_M_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_xeqm_M_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeqm_M_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_xeqm_Ma_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeqm_Ma_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_xeqm_Ma_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeqm_Ma_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_xeqm_Ma_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeqm_Ma_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_xeqm_Ma_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeqm_Ma_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_xeqm_pM_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeqm_pM_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_xeqm_pM_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeqm_pM_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_xeqm_pM_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeqm_pM_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_xeqm_pM_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeqm_pM_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, true>>("D3_lmult_M01", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_xeqm_pMa_times_M(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeqm_pMa_times_M");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_xeqm_pMa_times_pM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeqm_pMa_times_pM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_xeqm_pMa_times_Ma(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeqm_pMa_times_Ma");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_xeqm_pMa_times_pMa(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ * a, QLA_D3_ColorMatrix *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D3_M_xeqm_pMa_times_pMa");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, true>>("D3_lmult_M11", r, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_eq_M_times_xM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_M_eq_M_times_xM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_eq_Ma_times_xM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_M_eq_Ma_times_xM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D3_M_peq_M_times_xM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_M_peq_M_times_xM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_peq_Ma_times_xM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_M_peq_Ma_times_xM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D3_M_meq_M_times_xM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_M_meq_M_times_xM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_meq_Ma_times_xM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_M_meq_Ma_times_xM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D3_M_eqm_M_times_xM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_M_eqm_M_times_xM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, false, false>>("D3_lmult_M00", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D3_M_eqm_Ma_times_xM(QLA_D3_ColorMatrix *__restrict__ r, QLA_D3_ColorMatrix *__restrict__ a, QLA_D3_ColorMatrix *__restrict__ b, int * jb, int n) {
  QLAB_TRACE("QLA_D3_M_eqm_Ma_times_xM");
  qlab::api_map<qlab::LMultOp<double, 3, 3, true, false>>("D3_lmult_M10", r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, qlab::EQM);
}

}  // extern "C"
