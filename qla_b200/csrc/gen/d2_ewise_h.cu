// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA D2 ewise_h entry points (extern "C"), reference: lib/perl/build_qla.pl:403-469, 1256-1420 (element-wise families)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_ncolor.cuh"
#include "../qla_random.cuh"

extern "C" {
QLAB_EXPORT void QLA_D2_H_veq_c_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_c_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_c_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_c_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_C_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_C_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_C_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_C_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_pC_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_pC_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_pC_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_pC_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_Ca_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_Ca_times_H");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_Ca_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_Ca_times_pH");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_pCa_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_pCa_times_H");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_pCa_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_pCa_times_pH");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_R_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_R_times_H");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_R_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_R_times_pH");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_pR_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_pR_times_H");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_pR_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_pR_times_pH");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_conj_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_H_veq_conj_H");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_conj_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_H_veq_conj_pH");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_i_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_H_veq_i_H");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_i_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_H_veq_i_pH");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_vpeq_c_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_vpeq_c_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_vpeq_c_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_vpeq_c_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_vpeq_C_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_vpeq_C_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_vpeq_C_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_vpeq_C_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_vpeq_pC_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_vpeq_pC_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_vpeq_pC_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_vpeq_pC_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_vpeq_Ca_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_vpeq_Ca_times_H");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_vpeq_Ca_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_vpeq_Ca_times_pH");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_vpeq_pCa_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_vpeq_pCa_times_H");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_vpeq_pCa_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_vpeq_pCa_times_pH");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_vpeq_R_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_vpeq_R_times_H");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_vpeq_R_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_vpeq_R_times_pH");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_vpeq_pR_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_vpeq_pR_times_H");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_vpeq_pR_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_vpeq_pR_times_pH");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_vpeq_conj_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_H_vpeq_conj_H");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_vpeq_conj_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_H_vpeq_conj_pH");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_vpeq_i_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_H_vpeq_i_H");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_vpeq_i_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_H_vpeq_i_pH");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_vmeq_c_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_vmeq_c_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_vmeq_c_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_vmeq_c_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_vmeq_C_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_vmeq_C_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_vmeq_C_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_vmeq_C_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_vmeq_pC_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_vmeq_pC_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_vmeq_pC_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_vmeq_pC_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_vmeq_Ca_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_vmeq_Ca_times_H");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_vmeq_Ca_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_vmeq_Ca_times_pH");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_vmeq_pCa_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_vmeq_pCa_times_H");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_vmeq_pCa_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_vmeq_pCa_times_pH");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_vmeq_R_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_vmeq_R_times_H");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_vmeq_R_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_vmeq_R_times_pH");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_vmeq_pR_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_vmeq_pR_times_H");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_vmeq_pR_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_vmeq_pR_times_pH");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_vmeq_conj_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_H_vmeq_conj_H");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_vmeq_conj_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_H_vmeq_conj_pH");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_vmeq_i_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_H_vmeq_i_H");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_vmeq_i_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_H_vmeq_i_pH");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_veqm_c_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_veqm_c_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_veqm_c_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_veqm_c_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_veqm_C_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_veqm_C_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_veqm_C_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_veqm_C_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_veqm_pC_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_veqm_pC_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_veqm_pC_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_veqm_pC_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_veqm_Ca_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_veqm_Ca_times_H");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_veqm_Ca_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_veqm_Ca_times_pH");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_veqm_pCa_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_veqm_pCa_times_H");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_veqm_pCa_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_veqm_pCa_times_pH");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_veqm_R_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_veqm_R_times_H");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_veqm_R_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_veqm_R_times_pH");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_veqm_pR_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_veqm_pR_times_H");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_veqm_pR_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_veqm_pR_times_pH");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_veqm_conj_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_H_veqm_conj_H");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_veqm_conj_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_H_veqm_conj_pH");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_veqm_i_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_H_veqm_i_H");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_veqm_i_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_H_veqm_i_pH");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_veq_H_plus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_H_plus_H");
  qlab::api_ew_n<double, qlab::EW_PLUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_r_times_H_plus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, QLA_D2_HalfFermion *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D2_H_veq_r_times_H_plus_H");
  qlab::api_ew_n<double, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_c_times_H_plus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, QLA_D2_HalfFermion *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D2_H_veq_c_times_H_plus_H");
  qlab::api_ew_n<double, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_H_minus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_H_minus_H");
  qlab::api_ew_n<double, qlab::EW_MINUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_r_times_H_minus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, QLA_D2_HalfFermion *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D2_H_veq_r_times_H_minus_H");
  qlab::api_ew_n<double, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_c_times_H_minus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, QLA_D2_HalfFermion *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D2_H_veq_c_times_H_minus_H");
  qlab::api_ew_n<double, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_H_plus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_H_plus_pH");
  qlab::api_ew_n<double, qlab::EW_PLUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_r_times_H_plus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, QLA_D2_HalfFermion *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D2_H_veq_r_times_H_plus_pH");
  qlab::api_ew_n<double, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_c_times_H_plus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, QLA_D2_HalfFermion *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D2_H_veq_c_times_H_plus_pH");
  qlab::api_ew_n<double, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_H_minus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_H_minus_pH");
  qlab::api_ew_n<double, qlab::EW_MINUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_r_times_H_minus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, QLA_D2_HalfFermion *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D2_H_veq_r_times_H_minus_pH");
  qlab::api_ew_n<double, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_c_times_H_minus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, QLA_D2_HalfFermion *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D2_H_veq_c_times_H_minus_pH");
  qlab::api_ew_n<double, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_pH_plus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_pH_plus_H");
  qlab::api_ew_n<double, qlab::EW_PLUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_r_times_pH_plus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, QLA_D2_HalfFermion *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D2_H_veq_r_times_pH_plus_H");
  qlab::api_ew_n<double, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_c_times_pH_plus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, QLA_D2_HalfFermion *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D2_H_veq_c_times_pH_plus_H");
  qlab::api_ew_n<double, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_pH_minus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_pH_minus_H");
  qlab::api_ew_n<double, qlab::EW_MINUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_r_times_pH_minus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, QLA_D2_HalfFermion *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D2_H_veq_r_times_pH_minus_H");
  qlab::api_ew_n<double, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_c_times_pH_minus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, QLA_D2_HalfFermion *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D2_H_veq_c_times_pH_minus_H");
  qlab::api_ew_n<double, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_pH_plus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_pH_plus_pH");
  qlab::api_ew_n<double, qlab::EW_PLUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_r_times_pH_plus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, QLA_D2_HalfFermion *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D2_H_veq_r_times_pH_plus_pH");
  qlab::api_ew_n<double, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_c_times_pH_plus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, QLA_D2_HalfFermion *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D2_H_veq_c_times_pH_plus_pH");
  qlab::api_ew_n<double, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_pH_minus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_H_veq_pH_minus_pH");
  qlab::api_ew_n<double, qlab::EW_MINUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_r_times_pH_minus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, QLA_D2_HalfFermion *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D2_H_veq_r_times_pH_minus_pH");
  qlab::api_ew_n<double, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_veq_c_times_pH_minus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, QLA_D2_HalfFermion *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D2_H_veq_c_times_pH_minus_pH");
  qlab::api_ew_n<double, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_c_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_c_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_c_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_c_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_C_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_C_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_C_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_C_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_pC_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_pC_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_pC_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_pC_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_Ca_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_Ca_times_H");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_Ca_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_Ca_times_pH");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_pCa_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_pCa_times_H");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_pCa_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_pCa_times_pH");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_R_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_R_times_H");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_R_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_R_times_pH");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_pR_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_pR_times_H");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_pR_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_pR_times_pH");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_conj_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_conj_H");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_conj_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_conj_pH");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_i_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_i_H");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_i_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_i_pH");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xpeq_c_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xpeq_c_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_xpeq_c_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xpeq_c_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_xpeq_C_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xpeq_C_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_xpeq_C_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xpeq_C_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_xpeq_pC_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xpeq_pC_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_xpeq_pC_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xpeq_pC_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_xpeq_Ca_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xpeq_Ca_times_H");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_xpeq_Ca_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xpeq_Ca_times_pH");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_xpeq_pCa_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xpeq_pCa_times_H");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_xpeq_pCa_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xpeq_pCa_times_pH");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_xpeq_R_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xpeq_R_times_H");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_xpeq_R_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xpeq_R_times_pH");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_xpeq_pR_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xpeq_pR_times_H");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_xpeq_pR_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xpeq_pR_times_pH");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_xpeq_conj_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xpeq_conj_H");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_xpeq_conj_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xpeq_conj_pH");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_xpeq_i_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xpeq_i_H");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_xpeq_i_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xpeq_i_pH");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_H_xmeq_c_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xmeq_c_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_xmeq_c_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xmeq_c_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_xmeq_C_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xmeq_C_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_xmeq_C_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xmeq_C_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_xmeq_pC_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xmeq_pC_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_xmeq_pC_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xmeq_pC_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_xmeq_Ca_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xmeq_Ca_times_H");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_xmeq_Ca_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xmeq_Ca_times_pH");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_xmeq_pCa_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xmeq_pCa_times_H");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_xmeq_pCa_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xmeq_pCa_times_pH");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_xmeq_R_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xmeq_R_times_H");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_xmeq_R_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xmeq_R_times_pH");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_xmeq_pR_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xmeq_pR_times_H");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_xmeq_pR_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xmeq_pR_times_pH");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_xmeq_conj_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xmeq_conj_H");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_xmeq_conj_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xmeq_conj_pH");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_xmeq_i_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xmeq_i_H");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_xmeq_i_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xmeq_i_pH");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_H_xeqm_c_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeqm_c_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_xeqm_c_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeqm_c_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_xeqm_C_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeqm_C_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_xeqm_C_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeqm_C_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_xeqm_pC_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeqm_pC_times_H");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_xeqm_pC_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeqm_pC_times_pH");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_xeqm_Ca_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeqm_Ca_times_H");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_xeqm_Ca_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeqm_Ca_times_pH");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_xeqm_pCa_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeqm_pCa_times_H");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_xeqm_pCa_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeqm_pCa_times_pH");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_xeqm_R_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeqm_R_times_H");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_xeqm_R_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeqm_R_times_pH");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_xeqm_pR_times_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeqm_pR_times_H");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_xeqm_pR_times_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeqm_pR_times_pH");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_xeqm_conj_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeqm_conj_H");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_xeqm_conj_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeqm_conj_pH");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_xeqm_i_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeqm_i_H");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_xeqm_i_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeqm_i_pH");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_H_xeq_H_plus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_H_plus_H");
  qlab::api_ew_n<double, qlab::EW_PLUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_r_times_H_plus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, QLA_D2_HalfFermion *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_r_times_H_plus_H");
  qlab::api_ew_n<double, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_c_times_H_plus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, QLA_D2_HalfFermion *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_c_times_H_plus_H");
  qlab::api_ew_n<double, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_H_minus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_H_minus_H");
  qlab::api_ew_n<double, qlab::EW_MINUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_r_times_H_minus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, QLA_D2_HalfFermion *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_r_times_H_minus_H");
  qlab::api_ew_n<double, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_c_times_H_minus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, QLA_D2_HalfFermion *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_c_times_H_minus_H");
  qlab::api_ew_n<double, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_H_plus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_H_plus_pH");
  qlab::api_ew_n<double, qlab::EW_PLUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_r_times_H_plus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, QLA_D2_HalfFermion *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_r_times_H_plus_pH");
  qlab::api_ew_n<double, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_c_times_H_plus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, QLA_D2_HalfFermion *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_c_times_H_plus_pH");
  qlab::api_ew_n<double, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_H_minus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_H_minus_pH");
  qlab::api_ew_n<double, qlab::EW_MINUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_r_times_H_minus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, QLA_D2_HalfFermion *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_r_times_H_minus_pH");
  qlab::api_ew_n<double, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_c_times_H_minus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ b, QLA_D2_HalfFermion *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_c_times_H_minus_pH");
  qlab::api_ew_n<double, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_pH_plus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_pH_plus_H");
  qlab::api_ew_n<double, qlab::EW_PLUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_r_times_pH_plus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, QLA_D2_HalfFermion *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_r_times_pH_plus_H");
  qlab::api_ew_n<double, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_c_times_pH_plus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, QLA_D2_HalfFermion *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_c_times_pH_plus_H");
  qlab::api_ew_n<double, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_pH_minus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_pH_minus_H");
  qlab::api_ew_n<double, qlab::EW_MINUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_r_times_pH_minus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, QLA_D2_HalfFermion *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_r_times_pH_minus_H");
  qlab::api_ew_n<double, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_c_times_pH_minus_H(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, QLA_D2_HalfFermion *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_c_times_pH_minus_H");
  qlab::api_ew_n<double, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_pH_plus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_pH_plus_pH");
  qlab::api_ew_n<double, qlab::EW_PLUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_r_times_pH_plus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, QLA_D2_HalfFermion *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_r_times_pH_plus_pH");
  qlab::api_ew_n<double, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_c_times_pH_plus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, QLA_D2_HalfFermion *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_c_times_pH_plus_pH");
  qlab::api_ew_n<double, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_pH_minus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D2_HalfFermion *__restrict__ * a, QLA_D2_HalfFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_pH_minus_pH");
  qlab::api_ew_n<double, qlab::EW_MINUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 2 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_r_times_pH_minus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, QLA_D2_HalfFermion *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_r_times_pH_minus_pH");
  qlab::api_ew_n<double, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_H_xeq_c_times_pH_minus_pH(QLA_D2_HalfFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_HalfFermion *__restrict__ * b, QLA_D2_HalfFermion *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D2_H_xeq_c_times_pH_minus_pH");
  qlab::api_ew_n<double, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 2 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

}  // extern "C"
