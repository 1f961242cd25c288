// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA I int entry points (extern "C"), reference: lib/perl/build_qla.pl:1932-2082 (integer fields)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_int.cuh"

extern "C" {
QLAB_EXPORT void QLA_I_veq_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, int n) {
  QLAB_TRACE("QLA_I_veq_I");
  qlab::api_int("I_int", qlab::IC_COPY, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, 1, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_I_times_I");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_I_times_pI");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_i_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_i_times_I");
  qlab::api_int("I_int", qlab::IC_S_TIMES, qlab::EQ, (int*)r, (const int*)a, qlab::op_contig(b), qlab::Opnd{}, qlab::Opnd{}, 1, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_I_veq_pI");
  qlab::api_int("I_int", qlab::IC_COPY, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, 1, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_times_I");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_times_pI");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_i_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_i_times_pI");
  qlab::api_int("I_int", qlab::IC_S_TIMES, qlab::EQ, (int*)r, (const int*)a, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, qlab::Opnd{}, 1, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_i(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, int n) {
  QLAB_TRACE("QLA_I_veq_i");
  qlab::api_int("I_int", qlab::IC_S, qlab::EQ, (int*)r, (const int*)a, qlab::Opnd{}, qlab::Opnd{}, qlab::Opnd{}, 0, nullptr, n);
}

QLAB_EXPORT void QLA_I_vpeq_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, int n) {
  QLAB_TRACE("QLA_I_vpeq_I");
  qlab::api_int("I_int", qlab::IC_COPY, qlab::PEQ, (int*)r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, 1, nullptr, n);
}

QLAB_EXPORT void QLA_I_vpeq_I_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_vpeq_I_times_I");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::PEQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_vpeq_I_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_vpeq_I_times_pI");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::PEQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_vpeq_i_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_vpeq_i_times_I");
  qlab::api_int("I_int", qlab::IC_S_TIMES, qlab::PEQ, (int*)r, (const int*)a, qlab::op_contig(b), qlab::Opnd{}, qlab::Opnd{}, 1, nullptr, n);
}

QLAB_EXPORT void QLA_I_vpeq_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_I_vpeq_pI");
  qlab::api_int("I_int", qlab::IC_COPY, qlab::PEQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, 1, nullptr, n);
}

QLAB_EXPORT void QLA_I_vpeq_pI_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_vpeq_pI_times_I");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::PEQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_vpeq_pI_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_vpeq_pI_times_pI");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::PEQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_vpeq_i_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_vpeq_i_times_pI");
  qlab::api_int("I_int", qlab::IC_S_TIMES, qlab::PEQ, (int*)r, (const int*)a, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, qlab::Opnd{}, 1, nullptr, n);
}

QLAB_EXPORT void QLA_I_vpeq_i(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, int n) {
  QLAB_TRACE("QLA_I_vpeq_i");
  qlab::api_int("I_int", qlab::IC_S, qlab::PEQ, (int*)r, (const int*)a, qlab::Opnd{}, qlab::Opnd{}, qlab::Opnd{}, 0, nullptr, n);
}

QLAB_EXPORT void QLA_I_vmeq_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, int n) {
  QLAB_TRACE("QLA_I_vmeq_I");
  qlab::api_int("I_int", qlab::IC_COPY, qlab::MEQ, (int*)r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, 1, nullptr, n);
}

QLAB_EXPORT void QLA_I_vmeq_I_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_vmeq_I_times_I");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::MEQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_vmeq_I_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_vmeq_I_times_pI");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::MEQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_vmeq_i_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_vmeq_i_times_I");
  qlab::api_int("I_int", qlab::IC_S_TIMES, qlab::MEQ, (int*)r, (const int*)a, qlab::op_contig(b), qlab::Opnd{}, qlab::Opnd{}, 1, nullptr, n);
}

QLAB_EXPORT void QLA_I_vmeq_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_I_vmeq_pI");
  qlab::api_int("I_int", qlab::IC_COPY, qlab::MEQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, 1, nullptr, n);
}

QLAB_EXPORT void QLA_I_vmeq_pI_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_vmeq_pI_times_I");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::MEQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_vmeq_pI_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_vmeq_pI_times_pI");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::MEQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_vmeq_i_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_vmeq_i_times_pI");
  qlab::api_int("I_int", qlab::IC_S_TIMES, qlab::MEQ, (int*)r, (const int*)a, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, qlab::Opnd{}, 1, nullptr, n);
}

QLAB_EXPORT void QLA_I_vmeq_i(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, int n) {
  QLAB_TRACE("QLA_I_vmeq_i");
  qlab::api_int("I_int", qlab::IC_S, qlab::MEQ, (int*)r, (const int*)a, qlab::Opnd{}, qlab::Opnd{}, qlab::Opnd{}, 0, nullptr, n);
}

QLAB_EXPORT void QLA_I_veqm_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, int n) {
  QLAB_TRACE("QLA_I_veqm_I");
  qlab::api_int("I_int", qlab::IC_COPY, qlab::EQM, (int*)r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, 1, nullptr, n);
}

QLAB_EXPORT void QLA_I_veqm_I_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veqm_I_times_I");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::EQM, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veqm_I_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veqm_I_times_pI");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::EQM, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veqm_i_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veqm_i_times_I");
  qlab::api_int("I_int", qlab::IC_S_TIMES, qlab::EQM, (int*)r, (const int*)a, qlab::op_contig(b), qlab::Opnd{}, qlab::Opnd{}, 1, nullptr, n);
}

QLAB_EXPORT void QLA_I_veqm_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_I_veqm_pI");
  qlab::api_int("I_int", qlab::IC_COPY, qlab::EQM, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, 1, nullptr, n);
}

QLAB_EXPORT void QLA_I_veqm_pI_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veqm_pI_times_I");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::EQM, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veqm_pI_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veqm_pI_times_pI");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::EQM, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veqm_i_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veqm_i_times_pI");
  qlab::api_int("I_int", qlab::IC_S_TIMES, qlab::EQM, (int*)r, (const int*)a, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, qlab::Opnd{}, 1, nullptr, n);
}

QLAB_EXPORT void QLA_I_veqm_i(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, int n) {
  QLAB_TRACE("QLA_I_veqm_i");
  qlab::api_int("I_int", qlab::IC_S, qlab::EQM, (int*)r, (const int*)a, qlab::Opnd{}, qlab::Opnd{}, qlab::Opnd{}, 0, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_and_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_I_and_I");
  qlab::api_int("I_int", qlab::IC_AND, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_and_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_I_and_pI");
  qlab::api_int("I_int", qlab::IC_AND, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_and_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_and_I");
  qlab::api_int("I_int", qlab::IC_AND, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_and_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_and_pI");
  qlab::api_int("I_int", qlab::IC_AND, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_divide_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_I_divide_I");
  qlab::api_int("I_int", qlab::IC_DIVIDE, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_divide_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_I_divide_pI");
  qlab::api_int("I_int", qlab::IC_DIVIDE, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_divide_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_divide_I");
  qlab::api_int("I_int", qlab::IC_DIVIDE, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_divide_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_divide_pI");
  qlab::api_int("I_int", qlab::IC_DIVIDE, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_eq_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_I_eq_I");
  qlab::api_int("I_int", qlab::IC_EQ, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_eq_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_I_eq_pI");
  qlab::api_int("I_int", qlab::IC_EQ, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_eq_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_eq_I");
  qlab::api_int("I_int", qlab::IC_EQ, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_eq_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_eq_pI");
  qlab::api_int("I_int", qlab::IC_EQ, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_ge_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_I_ge_I");
  qlab::api_int("I_int", qlab::IC_GE, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_ge_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_I_ge_pI");
  qlab::api_int("I_int", qlab::IC_GE, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_ge_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_ge_I");
  qlab::api_int("I_int", qlab::IC_GE, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_ge_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_ge_pI");
  qlab::api_int("I_int", qlab::IC_GE, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_gt_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_I_gt_I");
  qlab::api_int("I_int", qlab::IC_GT, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_gt_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_I_gt_pI");
  qlab::api_int("I_int", qlab::IC_GT, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_gt_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_gt_I");
  qlab::api_int("I_int", qlab::IC_GT, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_gt_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_gt_pI");
  qlab::api_int("I_int", qlab::IC_GT, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_le_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_I_le_I");
  qlab::api_int("I_int", qlab::IC_LE, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_le_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_I_le_pI");
  qlab::api_int("I_int", qlab::IC_LE, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_le_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_le_I");
  qlab::api_int("I_int", qlab::IC_LE, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_le_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_le_pI");
  qlab::api_int("I_int", qlab::IC_LE, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_lshift_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_I_lshift_I");
  qlab::api_int("I_int", qlab::IC_LSHIFT, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_lshift_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_I_lshift_pI");
  qlab::api_int("I_int", qlab::IC_LSHIFT, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_lshift_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_lshift_I");
  qlab::api_int("I_int", qlab::IC_LSHIFT, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_lshift_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_lshift_pI");
  qlab::api_int("I_int", qlab::IC_LSHIFT, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_lt_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_I_lt_I");
  qlab::api_int("I_int", qlab::IC_LT, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_lt_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_I_lt_pI");
  qlab::api_int("I_int", qlab::IC_LT, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_lt_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_lt_I");
  qlab::api_int("I_int", qlab::IC_LT, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_lt_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_lt_pI");
  qlab::api_int("I_int", qlab::IC_LT, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_mask_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_I_mask_I");
  qlab::api_int("I_int", qlab::IC_MASK, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_mask_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_I_mask_pI");
  qlab::api_int("I_int", qlab::IC_MASK, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_mask_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_mask_I");
  qlab::api_int("I_int", qlab::IC_MASK, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_mask_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_mask_pI");
  qlab::api_int("I_int", qlab::IC_MASK, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_max_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_I_max_I");
  qlab::api_int("I_int", qlab::IC_MAX, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_max_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_I_max_pI");
  qlab::api_int("I_int", qlab::IC_MAX, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_max_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_max_I");
  qlab::api_int("I_int", qlab::IC_MAX, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_max_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_max_pI");
  qlab::api_int("I_int", qlab::IC_MAX, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_min_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_I_min_I");
  qlab::api_int("I_int", qlab::IC_MIN, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_min_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_I_min_pI");
  qlab::api_int("I_int", qlab::IC_MIN, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_min_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_min_I");
  qlab::api_int("I_int", qlab::IC_MIN, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_min_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_min_pI");
  qlab::api_int("I_int", qlab::IC_MIN, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_minus_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_I_minus_I");
  qlab::api_int("I_int", qlab::IC_MINUS, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_minus_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_I_minus_pI");
  qlab::api_int("I_int", qlab::IC_MINUS, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_minus_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_minus_I");
  qlab::api_int("I_int", qlab::IC_MINUS, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_minus_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_minus_pI");
  qlab::api_int("I_int", qlab::IC_MINUS, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_mod_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_I_mod_I");
  qlab::api_int("I_int", qlab::IC_MOD, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_mod_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_I_mod_pI");
  qlab::api_int("I_int", qlab::IC_MOD, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_mod_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_mod_I");
  qlab::api_int("I_int", qlab::IC_MOD, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_mod_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_mod_pI");
  qlab::api_int("I_int", qlab::IC_MOD, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_ne_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_I_ne_I");
  qlab::api_int("I_int", qlab::IC_NE, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_ne_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_I_ne_pI");
  qlab::api_int("I_int", qlab::IC_NE, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_ne_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_ne_I");
  qlab::api_int("I_int", qlab::IC_NE, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_ne_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_ne_pI");
  qlab::api_int("I_int", qlab::IC_NE, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_or_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_I_or_I");
  qlab::api_int("I_int", qlab::IC_OR, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_or_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_I_or_pI");
  qlab::api_int("I_int", qlab::IC_OR, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_or_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_or_I");
  qlab::api_int("I_int", qlab::IC_OR, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_or_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_or_pI");
  qlab::api_int("I_int", qlab::IC_OR, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_plus_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_I_plus_I");
  qlab::api_int("I_int", qlab::IC_PLUS, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_plus_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_I_plus_pI");
  qlab::api_int("I_int", qlab::IC_PLUS, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_plus_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_plus_I");
  qlab::api_int("I_int", qlab::IC_PLUS, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_plus_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_plus_pI");
  qlab::api_int("I_int", qlab::IC_PLUS, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_rshift_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_I_rshift_I");
  qlab::api_int("I_int", qlab::IC_RSHIFT, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_rshift_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_I_rshift_pI");
  qlab::api_int("I_int", qlab::IC_RSHIFT, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_rshift_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_rshift_I");
  qlab::api_int("I_int", qlab::IC_RSHIFT, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_rshift_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_rshift_pI");
  qlab::api_int("I_int", qlab::IC_RSHIFT, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_xor_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_I_xor_I");
  qlab::api_int("I_int", qlab::IC_XOR, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_I_xor_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_I_xor_pI");
  qlab::api_int("I_int", qlab::IC_XOR, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_xor_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_xor_I");
  qlab::api_int("I_int", qlab::IC_XOR, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_pI_xor_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_I_veq_pI_xor_pI");
  qlab::api_int("I_int", qlab::IC_XOR, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_i_times_I_plus_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, QLA_Int *__restrict__ c, int n) {
  QLAB_TRACE("QLA_I_veq_i_times_I_plus_I");
  qlab::api_int("I_int", qlab::IC_S_TIMES_PLUS, qlab::EQ, (int*)r, (const int*)a, qlab::op_contig(b), qlab::op_contig(c), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_i_times_I_plus_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, QLA_Int *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_I_veq_i_times_I_plus_pI");
  qlab::api_int("I_int", qlab::IC_S_TIMES_PLUS, qlab::EQ, (int*)r, (const int*)a, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_i_times_I_minus_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, QLA_Int *__restrict__ c, int n) {
  QLAB_TRACE("QLA_I_veq_i_times_I_minus_I");
  qlab::api_int("I_int", qlab::IC_S_TIMES_MINUS, qlab::EQ, (int*)r, (const int*)a, qlab::op_contig(b), qlab::op_contig(c), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_i_times_I_minus_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, QLA_Int *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_I_veq_i_times_I_minus_pI");
  qlab::api_int("I_int", qlab::IC_S_TIMES_MINUS, qlab::EQ, (int*)r, (const int*)a, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_not_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, int n) {
  QLAB_TRACE("QLA_I_veq_not_I");
  qlab::api_int("I_int", qlab::IC_NOT, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, 1, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_i_times_pI_plus_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, QLA_Int *__restrict__ c, int n) {
  QLAB_TRACE("QLA_I_veq_i_times_pI_plus_I");
  qlab::api_int("I_int", qlab::IC_S_TIMES_PLUS, qlab::EQ, (int*)r, (const int*)a, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_i_times_pI_plus_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, QLA_Int *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_I_veq_i_times_pI_plus_pI");
  qlab::api_int("I_int", qlab::IC_S_TIMES_PLUS, qlab::EQ, (int*)r, (const int*)a, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_i_times_pI_minus_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, QLA_Int *__restrict__ c, int n) {
  QLAB_TRACE("QLA_I_veq_i_times_pI_minus_I");
  qlab::api_int("I_int", qlab::IC_S_TIMES_MINUS, qlab::EQ, (int*)r, (const int*)a, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_i_times_pI_minus_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, QLA_Int *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_I_veq_i_times_pI_minus_pI");
  qlab::api_int("I_int", qlab::IC_S_TIMES_MINUS, qlab::EQ, (int*)r, (const int*)a, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), qlab::Opnd{}, 2, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_not_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_I_veq_not_pI");
  qlab::api_int("I_int", qlab::IC_NOT, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, 1, nullptr, n);
}

QLAB_EXPORT void QLA_I_veq_zero(QLA_Int *__restrict__ r, int n) {
  QLAB_TRACE("QLA_I_veq_zero");
  qlab::api_int("I_int", qlab::IC_ZERO, qlab::EQ, (int*)r, nullptr, qlab::Opnd{}, qlab::Opnd{}, qlab::Opnd{}, 0, nullptr, n);
}

QLAB_EXPORT void QLA_I_xeq_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I");
  qlab::api_int("I_int", qlab::IC_COPY, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, 1, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_times_I");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_times_pI");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_i_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_i_times_I");
  qlab::api_int("I_int", qlab::IC_S_TIMES, qlab::EQ, (int*)r, (const int*)a, qlab::op_contig(b), qlab::Opnd{}, qlab::Opnd{}, 1, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI");
  qlab::api_int("I_int", qlab::IC_COPY, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, 1, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_times_I");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_times_pI");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_i_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_i_times_pI");
  qlab::api_int("I_int", qlab::IC_S_TIMES, qlab::EQ, (int*)r, (const int*)a, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, qlab::Opnd{}, 1, index, n);
}

QLAB_EXPORT void QLA_I_xeq_i(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_i");
  qlab::api_int("I_int", qlab::IC_S, qlab::EQ, (int*)r, (const int*)a, qlab::Opnd{}, qlab::Opnd{}, qlab::Opnd{}, 0, index, n);
}

QLAB_EXPORT void QLA_I_xpeq_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_I_xpeq_I");
  qlab::api_int("I_int", qlab::IC_COPY, qlab::PEQ, (int*)r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, 1, index, n);
}

QLAB_EXPORT void QLA_I_xpeq_I_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xpeq_I_times_I");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::PEQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xpeq_I_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xpeq_I_times_pI");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::PEQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xpeq_i_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xpeq_i_times_I");
  qlab::api_int("I_int", qlab::IC_S_TIMES, qlab::PEQ, (int*)r, (const int*)a, qlab::op_contig(b), qlab::Opnd{}, qlab::Opnd{}, 1, index, n);
}

QLAB_EXPORT void QLA_I_xpeq_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_I_xpeq_pI");
  qlab::api_int("I_int", qlab::IC_COPY, qlab::PEQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, 1, index, n);
}

QLAB_EXPORT void QLA_I_xpeq_pI_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xpeq_pI_times_I");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::PEQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xpeq_pI_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xpeq_pI_times_pI");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::PEQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xpeq_i_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xpeq_i_times_pI");
  qlab::api_int("I_int", qlab::IC_S_TIMES, qlab::PEQ, (int*)r, (const int*)a, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, qlab::Opnd{}, 1, index, n);
}

QLAB_EXPORT void QLA_I_xpeq_i(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_I_xpeq_i");
  qlab::api_int("I_int", qlab::IC_S, qlab::PEQ, (int*)r, (const int*)a, qlab::Opnd{}, qlab::Opnd{}, qlab::Opnd{}, 0, index, n);
}

QLAB_EXPORT void QLA_I_xmeq_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_I_xmeq_I");
  qlab::api_int("I_int", qlab::IC_COPY, qlab::MEQ, (int*)r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, 1, index, n);
}

QLAB_EXPORT void QLA_I_xmeq_I_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xmeq_I_times_I");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::MEQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xmeq_I_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xmeq_I_times_pI");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::MEQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xmeq_i_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xmeq_i_times_I");
  qlab::api_int("I_int", qlab::IC_S_TIMES, qlab::MEQ, (int*)r, (const int*)a, qlab::op_contig(b), qlab::Opnd{}, qlab::Opnd{}, 1, index, n);
}

QLAB_EXPORT void QLA_I_xmeq_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_I_xmeq_pI");
  qlab::api_int("I_int", qlab::IC_COPY, qlab::MEQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, 1, index, n);
}

QLAB_EXPORT void QLA_I_xmeq_pI_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xmeq_pI_times_I");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::MEQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xmeq_pI_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xmeq_pI_times_pI");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::MEQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xmeq_i_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xmeq_i_times_pI");
  qlab::api_int("I_int", qlab::IC_S_TIMES, qlab::MEQ, (int*)r, (const int*)a, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, qlab::Opnd{}, 1, index, n);
}

QLAB_EXPORT void QLA_I_xmeq_i(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_I_xmeq_i");
  qlab::api_int("I_int", qlab::IC_S, qlab::MEQ, (int*)r, (const int*)a, qlab::Opnd{}, qlab::Opnd{}, qlab::Opnd{}, 0, index, n);
}

QLAB_EXPORT void QLA_I_xeqm_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_I_xeqm_I");
  qlab::api_int("I_int", qlab::IC_COPY, qlab::EQM, (int*)r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, 1, index, n);
}

QLAB_EXPORT void QLA_I_xeqm_I_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeqm_I_times_I");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::EQM, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeqm_I_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeqm_I_times_pI");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::EQM, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeqm_i_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeqm_i_times_I");
  qlab::api_int("I_int", qlab::IC_S_TIMES, qlab::EQM, (int*)r, (const int*)a, qlab::op_contig(b), qlab::Opnd{}, qlab::Opnd{}, 1, index, n);
}

QLAB_EXPORT void QLA_I_xeqm_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_I_xeqm_pI");
  qlab::api_int("I_int", qlab::IC_COPY, qlab::EQM, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, 1, index, n);
}

QLAB_EXPORT void QLA_I_xeqm_pI_times_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeqm_pI_times_I");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::EQM, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeqm_pI_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeqm_pI_times_pI");
  qlab::api_int("I_int", qlab::IC_TIMES, qlab::EQM, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeqm_i_times_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeqm_i_times_pI");
  qlab::api_int("I_int", qlab::IC_S_TIMES, qlab::EQM, (int*)r, (const int*)a, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, qlab::Opnd{}, 1, index, n);
}

QLAB_EXPORT void QLA_I_xeqm_i(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_I_xeqm_i");
  qlab::api_int("I_int", qlab::IC_S, qlab::EQM, (int*)r, (const int*)a, qlab::Opnd{}, qlab::Opnd{}, qlab::Opnd{}, 0, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_and_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_and_I");
  qlab::api_int("I_int", qlab::IC_AND, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_and_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_and_pI");
  qlab::api_int("I_int", qlab::IC_AND, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_and_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_and_I");
  qlab::api_int("I_int", qlab::IC_AND, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_and_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_and_pI");
  qlab::api_int("I_int", qlab::IC_AND, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_divide_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_divide_I");
  qlab::api_int("I_int", qlab::IC_DIVIDE, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_divide_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_divide_pI");
  qlab::api_int("I_int", qlab::IC_DIVIDE, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_divide_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_divide_I");
  qlab::api_int("I_int", qlab::IC_DIVIDE, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_divide_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_divide_pI");
  qlab::api_int("I_int", qlab::IC_DIVIDE, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_eq_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_eq_I");
  qlab::api_int("I_int", qlab::IC_EQ, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_eq_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_eq_pI");
  qlab::api_int("I_int", qlab::IC_EQ, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_eq_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_eq_I");
  qlab::api_int("I_int", qlab::IC_EQ, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_eq_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_eq_pI");
  qlab::api_int("I_int", qlab::IC_EQ, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_ge_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_ge_I");
  qlab::api_int("I_int", qlab::IC_GE, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_ge_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_ge_pI");
  qlab::api_int("I_int", qlab::IC_GE, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_ge_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_ge_I");
  qlab::api_int("I_int", qlab::IC_GE, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_ge_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_ge_pI");
  qlab::api_int("I_int", qlab::IC_GE, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_gt_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_gt_I");
  qlab::api_int("I_int", qlab::IC_GT, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_gt_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_gt_pI");
  qlab::api_int("I_int", qlab::IC_GT, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_gt_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_gt_I");
  qlab::api_int("I_int", qlab::IC_GT, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_gt_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_gt_pI");
  qlab::api_int("I_int", qlab::IC_GT, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_le_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_le_I");
  qlab::api_int("I_int", qlab::IC_LE, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_le_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_le_pI");
  qlab::api_int("I_int", qlab::IC_LE, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_le_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_le_I");
  qlab::api_int("I_int", qlab::IC_LE, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_le_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_le_pI");
  qlab::api_int("I_int", qlab::IC_LE, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_lshift_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_lshift_I");
  qlab::api_int("I_int", qlab::IC_LSHIFT, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_lshift_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_lshift_pI");
  qlab::api_int("I_int", qlab::IC_LSHIFT, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_lshift_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_lshift_I");
  qlab::api_int("I_int", qlab::IC_LSHIFT, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_lshift_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_lshift_pI");
  qlab::api_int("I_int", qlab::IC_LSHIFT, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_lt_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_lt_I");
  qlab::api_int("I_int", qlab::IC_LT, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_lt_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_lt_pI");
  qlab::api_int("I_int", qlab::IC_LT, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_lt_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_lt_I");
  qlab::api_int("I_int", qlab::IC_LT, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_lt_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_lt_pI");
  qlab::api_int("I_int", qlab::IC_LT, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_mask_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_mask_I");
  qlab::api_int("I_int", qlab::IC_MASK, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_mask_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_mask_pI");
  qlab::api_int("I_int", qlab::IC_MASK, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_mask_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_mask_I");
  qlab::api_int("I_int", qlab::IC_MASK, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_mask_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_mask_pI");
  qlab::api_int("I_int", qlab::IC_MASK, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_max_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_max_I");
  qlab::api_int("I_int", qlab::IC_MAX, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_max_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_max_pI");
  qlab::api_int("I_int", qlab::IC_MAX, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_max_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_max_I");
  qlab::api_int("I_int", qlab::IC_MAX, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_max_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_max_pI");
  qlab::api_int("I_int", qlab::IC_MAX, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_min_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_min_I");
  qlab::api_int("I_int", qlab::IC_MIN, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_min_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_min_pI");
  qlab::api_int("I_int", qlab::IC_MIN, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_min_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_min_I");
  qlab::api_int("I_int", qlab::IC_MIN, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_min_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_min_pI");
  qlab::api_int("I_int", qlab::IC_MIN, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_minus_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_minus_I");
  qlab::api_int("I_int", qlab::IC_MINUS, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_minus_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_minus_pI");
  qlab::api_int("I_int", qlab::IC_MINUS, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_minus_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_minus_I");
  qlab::api_int("I_int", qlab::IC_MINUS, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_minus_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_minus_pI");
  qlab::api_int("I_int", qlab::IC_MINUS, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_mod_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_mod_I");
  qlab::api_int("I_int", qlab::IC_MOD, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_mod_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_mod_pI");
  qlab::api_int("I_int", qlab::IC_MOD, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_mod_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_mod_I");
  qlab::api_int("I_int", qlab::IC_MOD, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_mod_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_mod_pI");
  qlab::api_int("I_int", qlab::IC_MOD, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_ne_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_ne_I");
  qlab::api_int("I_int", qlab::IC_NE, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_ne_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_ne_pI");
  qlab::api_int("I_int", qlab::IC_NE, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_ne_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_ne_I");
  qlab::api_int("I_int", qlab::IC_NE, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_ne_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_ne_pI");
  qlab::api_int("I_int", qlab::IC_NE, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_or_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_or_I");
  qlab::api_int("I_int", qlab::IC_OR, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_or_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_or_pI");
  qlab::api_int("I_int", qlab::IC_OR, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_or_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_or_I");
  qlab::api_int("I_int", qlab::IC_OR, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_or_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_or_pI");
  qlab::api_int("I_int", qlab::IC_OR, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_plus_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_plus_I");
  qlab::api_int("I_int", qlab::IC_PLUS, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_plus_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_plus_pI");
  qlab::api_int("I_int", qlab::IC_PLUS, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_plus_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_plus_I");
  qlab::api_int("I_int", qlab::IC_PLUS, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_plus_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_plus_pI");
  qlab::api_int("I_int", qlab::IC_PLUS, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_rshift_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_rshift_I");
  qlab::api_int("I_int", qlab::IC_RSHIFT, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_rshift_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_rshift_pI");
  qlab::api_int("I_int", qlab::IC_RSHIFT, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_rshift_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_rshift_I");
  qlab::api_int("I_int", qlab::IC_RSHIFT, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_rshift_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_rshift_pI");
  qlab::api_int("I_int", qlab::IC_RSHIFT, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_xor_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_xor_I");
  qlab::api_int("I_int", qlab::IC_XOR, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_I_xor_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_I_xor_pI");
  qlab::api_int("I_int", qlab::IC_XOR, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_xor_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_xor_I");
  qlab::api_int("I_int", qlab::IC_XOR, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_pI_xor_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, QLA_Int *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_pI_xor_pI");
  qlab::api_int("I_int", qlab::IC_XOR, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_i_times_I_plus_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, QLA_Int *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_i_times_I_plus_I");
  qlab::api_int("I_int", qlab::IC_S_TIMES_PLUS, qlab::EQ, (int*)r, (const int*)a, qlab::op_contig(b), qlab::op_contig(c), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_i_times_I_plus_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, QLA_Int *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_i_times_I_plus_pI");
  qlab::api_int("I_int", qlab::IC_S_TIMES_PLUS, qlab::EQ, (int*)r, (const int*)a, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_i_times_I_minus_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, QLA_Int *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_i_times_I_minus_I");
  qlab::api_int("I_int", qlab::IC_S_TIMES_MINUS, qlab::EQ, (int*)r, (const int*)a, qlab::op_contig(b), qlab::op_contig(c), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_i_times_I_minus_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ b, QLA_Int *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_i_times_I_minus_pI");
  qlab::api_int("I_int", qlab::IC_S_TIMES_MINUS, qlab::EQ, (int*)r, (const int*)a, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_not_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_not_I");
  qlab::api_int("I_int", qlab::IC_NOT, qlab::EQ, (int*)r, nullptr, qlab::op_contig(a), qlab::Opnd{}, qlab::Opnd{}, 1, index, n);
}

QLAB_EXPORT void QLA_I_xeq_i_times_pI_plus_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, QLA_Int *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_i_times_pI_plus_I");
  qlab::api_int("I_int", qlab::IC_S_TIMES_PLUS, qlab::EQ, (int*)r, (const int*)a, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_i_times_pI_plus_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, QLA_Int *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_i_times_pI_plus_pI");
  qlab::api_int("I_int", qlab::IC_S_TIMES_PLUS, qlab::EQ, (int*)r, (const int*)a, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_i_times_pI_minus_I(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, QLA_Int *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_i_times_pI_minus_I");
  qlab::api_int("I_int", qlab::IC_S_TIMES_MINUS, qlab::EQ, (int*)r, (const int*)a, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_i_times_pI_minus_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ a, QLA_Int *__restrict__ * b, QLA_Int *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_i_times_pI_minus_pI");
  qlab::api_int("I_int", qlab::IC_S_TIMES_MINUS, qlab::EQ, (int*)r, (const int*)a, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), qlab::Opnd{}, 2, index, n);
}

QLAB_EXPORT void QLA_I_xeq_not_pI(QLA_Int *__restrict__ r, QLA_Int *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_not_pI");
  qlab::api_int("I_int", qlab::IC_NOT, qlab::EQ, (int*)r, nullptr, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, qlab::Opnd{}, 1, index, n);
}

QLAB_EXPORT void QLA_I_xeq_zero(QLA_Int *__restrict__ r, int * index, int n) {
  QLAB_TRACE("QLA_I_xeq_zero");
  qlab::api_int("I_int", qlab::IC_ZERO, qlab::EQ, (int*)r, nullptr, qlab::Opnd{}, qlab::Opnd{}, qlab::Opnd{}, 0, index, n);
}

}  // extern "C"
