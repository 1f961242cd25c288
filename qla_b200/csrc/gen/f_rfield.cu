// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA F rfield entry points (extern "C"), reference: lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: elementary functions, arithmetic, comparisons, masks, conversions, reductions), include/qla_complex.h:110-140, 417-428, lib/cmath
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_scalar.cuh"

extern "C" {
QLAB_EXPORT void QLA_F_R_veq_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_R");
  qlab::api_scalar<float, qlab::SO_R_COPY>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_pR");
  qlab::api_scalar<float, qlab::SO_R_COPY>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_vpeq_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_vpeq_R");
  qlab::api_scalar<float, qlab::SO_R_COPY>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F_R_vpeq_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_vpeq_pR");
  qlab::api_scalar<float, qlab::SO_R_COPY>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F_R_vmeq_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_vmeq_R");
  qlab::api_scalar<float, qlab::SO_R_COPY>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F_R_vmeq_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_vmeq_pR");
  qlab::api_scalar<float, qlab::SO_R_COPY>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F_R_veqm_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veqm_R");
  qlab::api_scalar<float, qlab::SO_R_COPY>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F_R_veqm_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veqm_pR");
  qlab::api_scalar<float, qlab::SO_R_COPY>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F_R_xeq_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_R");
  qlab::api_scalar<float, qlab::SO_R_COPY>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pR");
  qlab::api_scalar<float, qlab::SO_R_COPY>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xpeq_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xpeq_R");
  qlab::api_scalar<float, qlab::SO_R_COPY>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F_R_xpeq_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xpeq_pR");
  qlab::api_scalar<float, qlab::SO_R_COPY>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F_R_xmeq_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xmeq_R");
  qlab::api_scalar<float, qlab::SO_R_COPY>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F_R_xmeq_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xmeq_pR");
  qlab::api_scalar<float, qlab::SO_R_COPY>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F_R_xeqm_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeqm_R");
  qlab::api_scalar<float, qlab::SO_R_COPY>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F_R_xeqm_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeqm_pR");
  qlab::api_scalar<float, qlab::SO_R_COPY>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F_R_veq_I(QLA_F_Real *__restrict__ r, QLA_Int *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_I");
  qlab::api_scalar<float, qlab::SO_R_FROM_I>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pI(QLA_F_Real *__restrict__ r, QLA_Int *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_pI");
  qlab::api_scalar<float, qlab::SO_R_FROM_I>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_I(QLA_F_Real *__restrict__ r, QLA_Int *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_I");
  qlab::api_scalar<float, qlab::SO_R_FROM_I>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pI(QLA_F_Real *__restrict__ r, QLA_Int *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pI");
  qlab::api_scalar<float, qlab::SO_R_FROM_I>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_r(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_r");
  qlab::api_scalar<float, qlab::SO_R_FILL>("F_scalar", r, a, qlab::Opnd{}, qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_vpeq_r(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_vpeq_r");
  qlab::api_scalar<float, qlab::SO_R_FILL>("F_scalar", r, a, qlab::Opnd{}, qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F_R_vmeq_r(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_vmeq_r");
  qlab::api_scalar<float, qlab::SO_R_FILL>("F_scalar", r, a, qlab::Opnd{}, qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F_R_veqm_r(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veqm_r");
  qlab::api_scalar<float, qlab::SO_R_FILL>("F_scalar", r, a, qlab::Opnd{}, qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F_R_xeq_r(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_r");
  qlab::api_scalar<float, qlab::SO_R_FILL>("F_scalar", r, a, qlab::Opnd{}, qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xpeq_r(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xpeq_r");
  qlab::api_scalar<float, qlab::SO_R_FILL>("F_scalar", r, a, qlab::Opnd{}, qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F_R_xmeq_r(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xmeq_r");
  qlab::api_scalar<float, qlab::SO_R_FILL>("F_scalar", r, a, qlab::Opnd{}, qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F_R_xeqm_r(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeqm_r");
  qlab::api_scalar<float, qlab::SO_R_FILL>("F_scalar", r, a, qlab::Opnd{}, qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F_R_veq_zero(QLA_F_Real *__restrict__ r, int n) {
  QLAB_TRACE("QLA_F_R_veq_zero");
  qlab::api_scalar<float, qlab::SO_R_ZERO>("F_scalar", r, nullptr, qlab::Opnd{}, qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_zero(QLA_F_Real *__restrict__ r, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_zero");
  qlab::api_scalar<float, qlab::SO_R_ZERO>("F_scalar", r, nullptr, qlab::Opnd{}, qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_R_mask_I(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veq_R_mask_I");
  qlab::api_scalar<float, qlab::SO_R_MASK>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_R_mask_pI(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veq_R_mask_pI");
  qlab::api_scalar<float, qlab::SO_R_MASK>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pR_mask_I(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veq_pR_mask_I");
  qlab::api_scalar<float, qlab::SO_R_MASK>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pR_mask_pI(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veq_pR_mask_pI");
  qlab::api_scalar<float, qlab::SO_R_MASK>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_R_mask_I(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_R_mask_I");
  qlab::api_scalar<float, qlab::SO_R_MASK>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_R_mask_pI(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_R_mask_pI");
  qlab::api_scalar<float, qlab::SO_R_MASK>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pR_mask_I(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pR_mask_I");
  qlab::api_scalar<float, qlab::SO_R_MASK>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pR_mask_pI(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pR_mask_pI");
  qlab::api_scalar<float, qlab::SO_R_MASK>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_R_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veq_R_times_R");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_R_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veq_R_times_pR");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pR_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veq_pR_times_R");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pR_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veq_pR_times_pR");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_vpeq_R_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_vpeq_R_times_R");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F_R_vpeq_R_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_vpeq_R_times_pR");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F_R_vpeq_pR_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_vpeq_pR_times_R");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F_R_vpeq_pR_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_vpeq_pR_times_pR");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F_R_vmeq_R_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_vmeq_R_times_R");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F_R_vmeq_R_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_vmeq_R_times_pR");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F_R_vmeq_pR_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_vmeq_pR_times_R");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F_R_vmeq_pR_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_vmeq_pR_times_pR");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F_R_veqm_R_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veqm_R_times_R");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F_R_veqm_R_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veqm_R_times_pR");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F_R_veqm_pR_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veqm_pR_times_R");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F_R_veqm_pR_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veqm_pR_times_pR");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F_R_xeq_R_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_R_times_R");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_R_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_R_times_pR");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pR_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pR_times_R");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pR_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pR_times_pR");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xpeq_R_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xpeq_R_times_R");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F_R_xpeq_R_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xpeq_R_times_pR");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F_R_xpeq_pR_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xpeq_pR_times_R");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F_R_xpeq_pR_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xpeq_pR_times_pR");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F_R_xmeq_R_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xmeq_R_times_R");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F_R_xmeq_R_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xmeq_R_times_pR");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F_R_xmeq_pR_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xmeq_pR_times_R");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F_R_xmeq_pR_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xmeq_pR_times_pR");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F_R_xeqm_R_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeqm_R_times_R");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F_R_xeqm_R_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeqm_R_times_pR");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F_R_xeqm_pR_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeqm_pR_times_R");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F_R_xeqm_pR_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeqm_pR_times_pR");
  qlab::api_scalar<float, qlab::SO_R_TIMES_R>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F_R_veq_r_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veq_r_times_R");
  qlab::api_scalar<float, qlab::SO_R_RTIMES>("F_scalar", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_r_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veq_r_times_pR");
  qlab::api_scalar<float, qlab::SO_R_RTIMES>("F_scalar", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_vpeq_r_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_vpeq_r_times_R");
  qlab::api_scalar<float, qlab::SO_R_RTIMES>("F_scalar", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F_R_vpeq_r_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_vpeq_r_times_pR");
  qlab::api_scalar<float, qlab::SO_R_RTIMES>("F_scalar", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F_R_vmeq_r_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_vmeq_r_times_R");
  qlab::api_scalar<float, qlab::SO_R_RTIMES>("F_scalar", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F_R_vmeq_r_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_vmeq_r_times_pR");
  qlab::api_scalar<float, qlab::SO_R_RTIMES>("F_scalar", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F_R_veqm_r_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veqm_r_times_R");
  qlab::api_scalar<float, qlab::SO_R_RTIMES>("F_scalar", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F_R_veqm_r_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veqm_r_times_pR");
  qlab::api_scalar<float, qlab::SO_R_RTIMES>("F_scalar", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F_R_xeq_r_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_r_times_R");
  qlab::api_scalar<float, qlab::SO_R_RTIMES>("F_scalar", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_r_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_r_times_pR");
  qlab::api_scalar<float, qlab::SO_R_RTIMES>("F_scalar", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xpeq_r_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xpeq_r_times_R");
  qlab::api_scalar<float, qlab::SO_R_RTIMES>("F_scalar", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F_R_xpeq_r_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xpeq_r_times_pR");
  qlab::api_scalar<float, qlab::SO_R_RTIMES>("F_scalar", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_F_R_xmeq_r_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xmeq_r_times_R");
  qlab::api_scalar<float, qlab::SO_R_RTIMES>("F_scalar", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F_R_xmeq_r_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xmeq_r_times_pR");
  qlab::api_scalar<float, qlab::SO_R_RTIMES>("F_scalar", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_F_R_xeqm_r_times_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeqm_r_times_R");
  qlab::api_scalar<float, qlab::SO_R_RTIMES>("F_scalar", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F_R_xeqm_r_times_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeqm_r_times_pR");
  qlab::api_scalar<float, qlab::SO_R_RTIMES>("F_scalar", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_F_R_veq_r_times_R_plus_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, QLA_F_Real *__restrict__ c, int n) {
  QLAB_TRACE("QLA_F_R_veq_r_times_R_plus_R");
  qlab::api_scalar<float, qlab::SO_R_RT_PLUS>("F_scalar", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_r_times_R_plus_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, QLA_F_Real *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_F_R_veq_r_times_R_plus_pR");
  qlab::api_scalar<float, qlab::SO_R_RT_PLUS>("F_scalar", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_r_times_pR_plus_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, QLA_F_Real *__restrict__ c, int n) {
  QLAB_TRACE("QLA_F_R_veq_r_times_pR_plus_R");
  qlab::api_scalar<float, qlab::SO_R_RT_PLUS>("F_scalar", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_r_times_pR_plus_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, QLA_F_Real *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_F_R_veq_r_times_pR_plus_pR");
  qlab::api_scalar<float, qlab::SO_R_RT_PLUS>("F_scalar", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_r_times_R_plus_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, QLA_F_Real *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_r_times_R_plus_R");
  qlab::api_scalar<float, qlab::SO_R_RT_PLUS>("F_scalar", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_r_times_R_plus_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, QLA_F_Real *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_r_times_R_plus_pR");
  qlab::api_scalar<float, qlab::SO_R_RT_PLUS>("F_scalar", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_r_times_pR_plus_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, QLA_F_Real *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_r_times_pR_plus_R");
  qlab::api_scalar<float, qlab::SO_R_RT_PLUS>("F_scalar", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_r_times_pR_plus_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, QLA_F_Real *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_r_times_pR_plus_pR");
  qlab::api_scalar<float, qlab::SO_R_RT_PLUS>("F_scalar", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_r_times_R_minus_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, QLA_F_Real *__restrict__ c, int n) {
  QLAB_TRACE("QLA_F_R_veq_r_times_R_minus_R");
  qlab::api_scalar<float, qlab::SO_R_RT_MINUS>("F_scalar", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_r_times_R_minus_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, QLA_F_Real *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_F_R_veq_r_times_R_minus_pR");
  qlab::api_scalar<float, qlab::SO_R_RT_MINUS>("F_scalar", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_r_times_pR_minus_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, QLA_F_Real *__restrict__ c, int n) {
  QLAB_TRACE("QLA_F_R_veq_r_times_pR_minus_R");
  qlab::api_scalar<float, qlab::SO_R_RT_MINUS>("F_scalar", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_r_times_pR_minus_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, QLA_F_Real *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_F_R_veq_r_times_pR_minus_pR");
  qlab::api_scalar<float, qlab::SO_R_RT_MINUS>("F_scalar", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_r_times_R_minus_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, QLA_F_Real *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_r_times_R_minus_R");
  qlab::api_scalar<float, qlab::SO_R_RT_MINUS>("F_scalar", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_r_times_R_minus_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, QLA_F_Real *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_r_times_R_minus_pR");
  qlab::api_scalar<float, qlab::SO_R_RT_MINUS>("F_scalar", r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_r_times_pR_minus_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, QLA_F_Real *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_r_times_pR_minus_R");
  qlab::api_scalar<float, qlab::SO_R_RT_MINUS>("F_scalar", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_r_times_pR_minus_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, QLA_F_Real *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_r_times_pR_minus_pR");
  qlab::api_scalar<float, qlab::SO_R_RT_MINUS>("F_scalar", r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_R_ldexp_I(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veq_R_ldexp_I");
  qlab::api_scalar<float, qlab::SO_R_LDEXP>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_R_ldexp_pI(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veq_R_ldexp_pI");
  qlab::api_scalar<float, qlab::SO_R_LDEXP>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pR_ldexp_I(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veq_pR_ldexp_I");
  qlab::api_scalar<float, qlab::SO_R_LDEXP>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pR_ldexp_pI(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veq_pR_ldexp_pI");
  qlab::api_scalar<float, qlab::SO_R_LDEXP>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_R_ldexp_I(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_R_ldexp_I");
  qlab::api_scalar<float, qlab::SO_R_LDEXP>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_R_ldexp_pI(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_R_ldexp_pI");
  qlab::api_scalar<float, qlab::SO_R_LDEXP>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pR_ldexp_I(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pR_ldexp_I");
  qlab::api_scalar<float, qlab::SO_R_LDEXP>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pR_ldexp_pI(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pR_ldexp_pI");
  qlab::api_scalar<float, qlab::SO_R_LDEXP>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_R_plus_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veq_R_plus_R");
  qlab::api_scalar<float, qlab::SO_R_PLUS>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_R_plus_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veq_R_plus_pR");
  qlab::api_scalar<float, qlab::SO_R_PLUS>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pR_plus_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veq_pR_plus_R");
  qlab::api_scalar<float, qlab::SO_R_PLUS>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pR_plus_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veq_pR_plus_pR");
  qlab::api_scalar<float, qlab::SO_R_PLUS>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_R_plus_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_R_plus_R");
  qlab::api_scalar<float, qlab::SO_R_PLUS>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_R_plus_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_R_plus_pR");
  qlab::api_scalar<float, qlab::SO_R_PLUS>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pR_plus_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pR_plus_R");
  qlab::api_scalar<float, qlab::SO_R_PLUS>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pR_plus_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pR_plus_pR");
  qlab::api_scalar<float, qlab::SO_R_PLUS>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_R_minus_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veq_R_minus_R");
  qlab::api_scalar<float, qlab::SO_R_MINUS>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_R_minus_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veq_R_minus_pR");
  qlab::api_scalar<float, qlab::SO_R_MINUS>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pR_minus_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veq_pR_minus_R");
  qlab::api_scalar<float, qlab::SO_R_MINUS>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pR_minus_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veq_pR_minus_pR");
  qlab::api_scalar<float, qlab::SO_R_MINUS>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_R_minus_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_R_minus_R");
  qlab::api_scalar<float, qlab::SO_R_MINUS>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_R_minus_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_R_minus_pR");
  qlab::api_scalar<float, qlab::SO_R_MINUS>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pR_minus_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pR_minus_R");
  qlab::api_scalar<float, qlab::SO_R_MINUS>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pR_minus_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pR_minus_pR");
  qlab::api_scalar<float, qlab::SO_R_MINUS>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_R_divide_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veq_R_divide_R");
  qlab::api_scalar<float, qlab::SO_R_DIVIDE>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_R_divide_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veq_R_divide_pR");
  qlab::api_scalar<float, qlab::SO_R_DIVIDE>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pR_divide_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veq_pR_divide_R");
  qlab::api_scalar<float, qlab::SO_R_DIVIDE>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pR_divide_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veq_pR_divide_pR");
  qlab::api_scalar<float, qlab::SO_R_DIVIDE>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_R_divide_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_R_divide_R");
  qlab::api_scalar<float, qlab::SO_R_DIVIDE>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_R_divide_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_R_divide_pR");
  qlab::api_scalar<float, qlab::SO_R_DIVIDE>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pR_divide_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pR_divide_R");
  qlab::api_scalar<float, qlab::SO_R_DIVIDE>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pR_divide_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pR_divide_pR");
  qlab::api_scalar<float, qlab::SO_R_DIVIDE>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_R_max_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veq_R_max_R");
  qlab::api_scalar<float, qlab::SO_R_MAX>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_R_max_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veq_R_max_pR");
  qlab::api_scalar<float, qlab::SO_R_MAX>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pR_max_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veq_pR_max_R");
  qlab::api_scalar<float, qlab::SO_R_MAX>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pR_max_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veq_pR_max_pR");
  qlab::api_scalar<float, qlab::SO_R_MAX>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_R_max_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_R_max_R");
  qlab::api_scalar<float, qlab::SO_R_MAX>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_R_max_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_R_max_pR");
  qlab::api_scalar<float, qlab::SO_R_MAX>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pR_max_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pR_max_R");
  qlab::api_scalar<float, qlab::SO_R_MAX>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pR_max_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pR_max_pR");
  qlab::api_scalar<float, qlab::SO_R_MAX>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_R_min_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veq_R_min_R");
  qlab::api_scalar<float, qlab::SO_R_MIN>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_R_min_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veq_R_min_pR");
  qlab::api_scalar<float, qlab::SO_R_MIN>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pR_min_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veq_pR_min_R");
  qlab::api_scalar<float, qlab::SO_R_MIN>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pR_min_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veq_pR_min_pR");
  qlab::api_scalar<float, qlab::SO_R_MIN>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_R_min_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_R_min_R");
  qlab::api_scalar<float, qlab::SO_R_MIN>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_R_min_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_R_min_pR");
  qlab::api_scalar<float, qlab::SO_R_MIN>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pR_min_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pR_min_R");
  qlab::api_scalar<float, qlab::SO_R_MIN>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pR_min_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pR_min_pR");
  qlab::api_scalar<float, qlab::SO_R_MIN>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_R_mod_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veq_R_mod_R");
  qlab::api_scalar<float, qlab::SO_R_MOD>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_R_mod_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veq_R_mod_pR");
  qlab::api_scalar<float, qlab::SO_R_MOD>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pR_mod_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veq_pR_mod_R");
  qlab::api_scalar<float, qlab::SO_R_MOD>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pR_mod_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veq_pR_mod_pR");
  qlab::api_scalar<float, qlab::SO_R_MOD>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_R_mod_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_R_mod_R");
  qlab::api_scalar<float, qlab::SO_R_MOD>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_R_mod_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_R_mod_pR");
  qlab::api_scalar<float, qlab::SO_R_MOD>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pR_mod_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pR_mod_R");
  qlab::api_scalar<float, qlab::SO_R_MOD>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pR_mod_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pR_mod_pR");
  qlab::api_scalar<float, qlab::SO_R_MOD>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_R_pow_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veq_R_pow_R");
  qlab::api_scalar<float, qlab::SO_R_POW>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_R_pow_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veq_R_pow_pR");
  qlab::api_scalar<float, qlab::SO_R_POW>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pR_pow_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veq_pR_pow_R");
  qlab::api_scalar<float, qlab::SO_R_POW>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pR_pow_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veq_pR_pow_pR");
  qlab::api_scalar<float, qlab::SO_R_POW>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_R_pow_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_R_pow_R");
  qlab::api_scalar<float, qlab::SO_R_POW>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_R_pow_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_R_pow_pR");
  qlab::api_scalar<float, qlab::SO_R_POW>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pR_pow_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pR_pow_R");
  qlab::api_scalar<float, qlab::SO_R_POW>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pR_pow_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pR_pow_pR");
  qlab::api_scalar<float, qlab::SO_R_POW>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_R_atan2_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veq_R_atan2_R");
  qlab::api_scalar<float, qlab::SO_R_ATAN2>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_R_atan2_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veq_R_atan2_pR");
  qlab::api_scalar<float, qlab::SO_R_ATAN2>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pR_atan2_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_R_veq_pR_atan2_R");
  qlab::api_scalar<float, qlab::SO_R_ATAN2>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_pR_atan2_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_R_veq_pR_atan2_pR");
  qlab::api_scalar<float, qlab::SO_R_ATAN2>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_R_atan2_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_R_atan2_R");
  qlab::api_scalar<float, qlab::SO_R_ATAN2>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_R_atan2_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_R_atan2_pR");
  qlab::api_scalar<float, qlab::SO_R_ATAN2>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pR_atan2_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pR_atan2_R");
  qlab::api_scalar<float, qlab::SO_R_ATAN2>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_pR_atan2_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_pR_atan2_pR");
  qlab::api_scalar<float, qlab::SO_R_ATAN2>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_sin_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_sin_R");
  qlab::api_scalar<float, qlab::SO_R_SIN>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_sin_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_sin_pR");
  qlab::api_scalar<float, qlab::SO_R_SIN>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_sin_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_sin_R");
  qlab::api_scalar<float, qlab::SO_R_SIN>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_sin_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_sin_pR");
  qlab::api_scalar<float, qlab::SO_R_SIN>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_cos_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_cos_R");
  qlab::api_scalar<float, qlab::SO_R_COS>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_cos_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_cos_pR");
  qlab::api_scalar<float, qlab::SO_R_COS>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_cos_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_cos_R");
  qlab::api_scalar<float, qlab::SO_R_COS>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_cos_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_cos_pR");
  qlab::api_scalar<float, qlab::SO_R_COS>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_tan_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_tan_R");
  qlab::api_scalar<float, qlab::SO_R_TAN>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_tan_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_tan_pR");
  qlab::api_scalar<float, qlab::SO_R_TAN>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_tan_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_tan_R");
  qlab::api_scalar<float, qlab::SO_R_TAN>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_tan_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_tan_pR");
  qlab::api_scalar<float, qlab::SO_R_TAN>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_asin_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_asin_R");
  qlab::api_scalar<float, qlab::SO_R_ASIN>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_asin_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_asin_pR");
  qlab::api_scalar<float, qlab::SO_R_ASIN>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_asin_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_asin_R");
  qlab::api_scalar<float, qlab::SO_R_ASIN>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_asin_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_asin_pR");
  qlab::api_scalar<float, qlab::SO_R_ASIN>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_acos_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_acos_R");
  qlab::api_scalar<float, qlab::SO_R_ACOS>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_acos_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_acos_pR");
  qlab::api_scalar<float, qlab::SO_R_ACOS>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_acos_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_acos_R");
  qlab::api_scalar<float, qlab::SO_R_ACOS>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_acos_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_acos_pR");
  qlab::api_scalar<float, qlab::SO_R_ACOS>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_atan_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_atan_R");
  qlab::api_scalar<float, qlab::SO_R_ATAN>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_atan_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_atan_pR");
  qlab::api_scalar<float, qlab::SO_R_ATAN>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_atan_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_atan_R");
  qlab::api_scalar<float, qlab::SO_R_ATAN>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_atan_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_atan_pR");
  qlab::api_scalar<float, qlab::SO_R_ATAN>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_sqrt_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_sqrt_R");
  qlab::api_scalar<float, qlab::SO_R_SQRT>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_sqrt_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_sqrt_pR");
  qlab::api_scalar<float, qlab::SO_R_SQRT>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_sqrt_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_sqrt_R");
  qlab::api_scalar<float, qlab::SO_R_SQRT>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_sqrt_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_sqrt_pR");
  qlab::api_scalar<float, qlab::SO_R_SQRT>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_fabs_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_fabs_R");
  qlab::api_scalar<float, qlab::SO_R_FABS>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_fabs_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_fabs_pR");
  qlab::api_scalar<float, qlab::SO_R_FABS>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_fabs_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_fabs_R");
  qlab::api_scalar<float, qlab::SO_R_FABS>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_fabs_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_fabs_pR");
  qlab::api_scalar<float, qlab::SO_R_FABS>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_exp_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_exp_R");
  qlab::api_scalar<float, qlab::SO_R_EXP>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_exp_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_exp_pR");
  qlab::api_scalar<float, qlab::SO_R_EXP>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_exp_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_exp_R");
  qlab::api_scalar<float, qlab::SO_R_EXP>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_exp_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_exp_pR");
  qlab::api_scalar<float, qlab::SO_R_EXP>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_log_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_log_R");
  qlab::api_scalar<float, qlab::SO_R_LOG>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_log_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_log_pR");
  qlab::api_scalar<float, qlab::SO_R_LOG>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_log_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_log_R");
  qlab::api_scalar<float, qlab::SO_R_LOG>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_log_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_log_pR");
  qlab::api_scalar<float, qlab::SO_R_LOG>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_log10_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_log10_R");
  qlab::api_scalar<float, qlab::SO_R_LOG10>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_log10_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_log10_pR");
  qlab::api_scalar<float, qlab::SO_R_LOG10>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_log10_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_log10_R");
  qlab::api_scalar<float, qlab::SO_R_LOG10>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_log10_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_log10_pR");
  qlab::api_scalar<float, qlab::SO_R_LOG10>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_sinh_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_sinh_R");
  qlab::api_scalar<float, qlab::SO_R_SINH>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_sinh_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_sinh_pR");
  qlab::api_scalar<float, qlab::SO_R_SINH>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_sinh_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_sinh_R");
  qlab::api_scalar<float, qlab::SO_R_SINH>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_sinh_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_sinh_pR");
  qlab::api_scalar<float, qlab::SO_R_SINH>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_cosh_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_cosh_R");
  qlab::api_scalar<float, qlab::SO_R_COSH>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_cosh_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_cosh_pR");
  qlab::api_scalar<float, qlab::SO_R_COSH>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_cosh_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_cosh_R");
  qlab::api_scalar<float, qlab::SO_R_COSH>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_cosh_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_cosh_pR");
  qlab::api_scalar<float, qlab::SO_R_COSH>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_tanh_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_tanh_R");
  qlab::api_scalar<float, qlab::SO_R_TANH>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_tanh_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_tanh_pR");
  qlab::api_scalar<float, qlab::SO_R_TANH>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_tanh_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_tanh_R");
  qlab::api_scalar<float, qlab::SO_R_TANH>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_tanh_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_tanh_pR");
  qlab::api_scalar<float, qlab::SO_R_TANH>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_ceil_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_ceil_R");
  qlab::api_scalar<float, qlab::SO_R_CEIL>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_ceil_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_ceil_pR");
  qlab::api_scalar<float, qlab::SO_R_CEIL>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_ceil_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_ceil_R");
  qlab::api_scalar<float, qlab::SO_R_CEIL>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_ceil_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_ceil_pR");
  qlab::api_scalar<float, qlab::SO_R_CEIL>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_floor_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_floor_R");
  qlab::api_scalar<float, qlab::SO_R_FLOOR>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_floor_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_floor_pR");
  qlab::api_scalar<float, qlab::SO_R_FLOOR>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_floor_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_floor_R");
  qlab::api_scalar<float, qlab::SO_R_FLOOR>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_floor_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_floor_pR");
  qlab::api_scalar<float, qlab::SO_R_FLOOR>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_sign_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_sign_R");
  qlab::api_scalar<float, qlab::SO_R_SIGN>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_sign_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_sign_pR");
  qlab::api_scalar<float, qlab::SO_R_SIGN>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_sign_R(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_sign_R");
  qlab::api_scalar<float, qlab::SO_R_SIGN>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_sign_pR(QLA_F_Real *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_sign_pR");
  qlab::api_scalar<float, qlab::SO_R_SIGN>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_re_C(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_re_C");
  qlab::api_scalar<float, qlab::SO_R_RE>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_re_pC(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_re_pC");
  qlab::api_scalar<float, qlab::SO_R_RE>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_re_C(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_re_C");
  qlab::api_scalar<float, qlab::SO_R_RE>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_re_pC(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_re_pC");
  qlab::api_scalar<float, qlab::SO_R_RE>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_im_C(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_im_C");
  qlab::api_scalar<float, qlab::SO_R_IM>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_im_pC(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_im_pC");
  qlab::api_scalar<float, qlab::SO_R_IM>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_im_C(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_im_C");
  qlab::api_scalar<float, qlab::SO_R_IM>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_im_pC(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_im_pC");
  qlab::api_scalar<float, qlab::SO_R_IM>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_norm_C(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_norm_C");
  qlab::api_scalar<float, qlab::SO_R_NORM>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_norm_pC(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_norm_pC");
  qlab::api_scalar<float, qlab::SO_R_NORM>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_norm_C(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_norm_C");
  qlab::api_scalar<float, qlab::SO_R_NORM>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_norm_pC(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_norm_pC");
  qlab::api_scalar<float, qlab::SO_R_NORM>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_arg_C(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_R_veq_arg_C");
  qlab::api_scalar<float, qlab::SO_R_ARG>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_veq_arg_pC(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_R_veq_arg_pC");
  qlab::api_scalar<float, qlab::SO_R_ARG>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_arg_C(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_arg_C");
  qlab::api_scalar<float, qlab::SO_R_ARG>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_R_xeq_arg_pC(QLA_F_Real *__restrict__ r, QLA_F_Complex *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_R_xeq_arg_pC");
  qlab::api_scalar<float, qlab::SO_R_ARG>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_R_eq_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_I_veq_R_eq_R");
  qlab::api_scalar<float, qlab::SO_I_EQ>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_R_eq_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_I_veq_R_eq_pR");
  qlab::api_scalar<float, qlab::SO_I_EQ>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_pR_eq_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_I_veq_pR_eq_R");
  qlab::api_scalar<float, qlab::SO_I_EQ>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_pR_eq_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_I_veq_pR_eq_pR");
  qlab::api_scalar<float, qlab::SO_I_EQ>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_R_eq_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_R_eq_R");
  qlab::api_scalar<float, qlab::SO_I_EQ>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_R_eq_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_R_eq_pR");
  qlab::api_scalar<float, qlab::SO_I_EQ>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_pR_eq_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_pR_eq_R");
  qlab::api_scalar<float, qlab::SO_I_EQ>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_pR_eq_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_pR_eq_pR");
  qlab::api_scalar<float, qlab::SO_I_EQ>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_R_ge_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_I_veq_R_ge_R");
  qlab::api_scalar<float, qlab::SO_I_GE>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_R_ge_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_I_veq_R_ge_pR");
  qlab::api_scalar<float, qlab::SO_I_GE>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_pR_ge_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_I_veq_pR_ge_R");
  qlab::api_scalar<float, qlab::SO_I_GE>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_pR_ge_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_I_veq_pR_ge_pR");
  qlab::api_scalar<float, qlab::SO_I_GE>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_R_ge_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_R_ge_R");
  qlab::api_scalar<float, qlab::SO_I_GE>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_R_ge_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_R_ge_pR");
  qlab::api_scalar<float, qlab::SO_I_GE>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_pR_ge_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_pR_ge_R");
  qlab::api_scalar<float, qlab::SO_I_GE>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_pR_ge_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_pR_ge_pR");
  qlab::api_scalar<float, qlab::SO_I_GE>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_R_gt_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_I_veq_R_gt_R");
  qlab::api_scalar<float, qlab::SO_I_GT>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_R_gt_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_I_veq_R_gt_pR");
  qlab::api_scalar<float, qlab::SO_I_GT>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_pR_gt_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_I_veq_pR_gt_R");
  qlab::api_scalar<float, qlab::SO_I_GT>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_pR_gt_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_I_veq_pR_gt_pR");
  qlab::api_scalar<float, qlab::SO_I_GT>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_R_gt_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_R_gt_R");
  qlab::api_scalar<float, qlab::SO_I_GT>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_R_gt_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_R_gt_pR");
  qlab::api_scalar<float, qlab::SO_I_GT>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_pR_gt_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_pR_gt_R");
  qlab::api_scalar<float, qlab::SO_I_GT>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_pR_gt_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_pR_gt_pR");
  qlab::api_scalar<float, qlab::SO_I_GT>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_R_le_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_I_veq_R_le_R");
  qlab::api_scalar<float, qlab::SO_I_LE>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_R_le_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_I_veq_R_le_pR");
  qlab::api_scalar<float, qlab::SO_I_LE>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_pR_le_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_I_veq_pR_le_R");
  qlab::api_scalar<float, qlab::SO_I_LE>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_pR_le_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_I_veq_pR_le_pR");
  qlab::api_scalar<float, qlab::SO_I_LE>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_R_le_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_R_le_R");
  qlab::api_scalar<float, qlab::SO_I_LE>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_R_le_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_R_le_pR");
  qlab::api_scalar<float, qlab::SO_I_LE>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_pR_le_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_pR_le_R");
  qlab::api_scalar<float, qlab::SO_I_LE>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_pR_le_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_pR_le_pR");
  qlab::api_scalar<float, qlab::SO_I_LE>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_R_lt_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_I_veq_R_lt_R");
  qlab::api_scalar<float, qlab::SO_I_LT>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_R_lt_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_I_veq_R_lt_pR");
  qlab::api_scalar<float, qlab::SO_I_LT>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_pR_lt_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_I_veq_pR_lt_R");
  qlab::api_scalar<float, qlab::SO_I_LT>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_pR_lt_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_I_veq_pR_lt_pR");
  qlab::api_scalar<float, qlab::SO_I_LT>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_R_lt_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_R_lt_R");
  qlab::api_scalar<float, qlab::SO_I_LT>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_R_lt_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_R_lt_pR");
  qlab::api_scalar<float, qlab::SO_I_LT>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_pR_lt_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_pR_lt_R");
  qlab::api_scalar<float, qlab::SO_I_LT>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_pR_lt_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_pR_lt_pR");
  qlab::api_scalar<float, qlab::SO_I_LT>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_R_ne_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_I_veq_R_ne_R");
  qlab::api_scalar<float, qlab::SO_I_NE>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_R_ne_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_I_veq_R_ne_pR");
  qlab::api_scalar<float, qlab::SO_I_NE>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_pR_ne_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int n) {
  QLAB_TRACE("QLA_F_I_veq_pR_ne_R");
  qlab::api_scalar<float, qlab::SO_I_NE>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_pR_ne_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_F_I_veq_pR_ne_pR");
  qlab::api_scalar<float, qlab::SO_I_NE>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_R_ne_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_R_ne_R");
  qlab::api_scalar<float, qlab::SO_I_NE>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_R_ne_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_R_ne_pR");
  qlab::api_scalar<float, qlab::SO_I_NE>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_pR_ne_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_pR_ne_R");
  qlab::api_scalar<float, qlab::SO_I_NE>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_pR_ne_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, QLA_F_Real *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_pR_ne_pR");
  qlab::api_scalar<float, qlab::SO_I_NE>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_round_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_I_veq_round_R");
  qlab::api_scalar<float, qlab::SO_I_ROUND>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_round_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_I_veq_round_pR");
  qlab::api_scalar<float, qlab::SO_I_ROUND>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_round_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_round_R");
  qlab::api_scalar<float, qlab::SO_I_ROUND>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_round_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_round_pR");
  qlab::api_scalar<float, qlab::SO_I_ROUND>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_trunc_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, int n) {
  QLAB_TRACE("QLA_F_I_veq_trunc_R");
  qlab::api_scalar<float, qlab::SO_I_TRUNC>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_veq_trunc_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_F_I_veq_trunc_pR");
  qlab::api_scalar<float, qlab::SO_I_TRUNC>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_trunc_R(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_trunc_R");
  qlab::api_scalar<float, qlab::SO_I_TRUNC>("F_scalar", r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_F_I_xeq_trunc_pR(QLA_Int *__restrict__ r, QLA_F_Real *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_F_I_xeq_trunc_pR");
  qlab::api_scalar<float, qlab::SO_I_TRUNC>("F_scalar", r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, index, n, qlab::EQ);
}

}  // extern "C"
