// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA D2 ewise_d entry points (extern "C"), reference: lib/perl/build_qla.pl:403-469, 1256-1420 (element-wise families)
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
#include "../qla_ncolor.cuh"
#include "../qla_random.cuh"

extern "C" {
QLAB_EXPORT void QLA_D2_D_veq_c_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_c_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_c_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_c_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_C_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_C_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_C_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_C_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_pC_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_pC_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_pC_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_pC_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_Ca_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_Ca_times_D");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_Ca_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_Ca_times_pD");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_pCa_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_pCa_times_D");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_pCa_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_pCa_times_pD");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_R_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_R_times_D");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_R_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_R_times_pD");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_pR_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_pR_times_D");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_pR_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_pR_times_pD");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_conj_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_D_veq_conj_D");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_conj_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_D_veq_conj_pD");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_i_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_D_veq_i_D");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_i_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_D_veq_i_pD");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_vpeq_c_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_vpeq_c_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_vpeq_c_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_vpeq_c_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_vpeq_C_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_vpeq_C_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_vpeq_C_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_vpeq_C_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_vpeq_pC_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_vpeq_pC_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_vpeq_pC_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_vpeq_pC_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_vpeq_Ca_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_vpeq_Ca_times_D");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_vpeq_Ca_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_vpeq_Ca_times_pD");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_vpeq_pCa_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_vpeq_pCa_times_D");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_vpeq_pCa_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_vpeq_pCa_times_pD");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_vpeq_R_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_vpeq_R_times_D");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_vpeq_R_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_vpeq_R_times_pD");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_vpeq_pR_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_vpeq_pR_times_D");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_vpeq_pR_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_vpeq_pR_times_pD");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_vpeq_conj_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_D_vpeq_conj_D");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_vpeq_conj_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_D_vpeq_conj_pD");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_vpeq_i_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_D_vpeq_i_D");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_vpeq_i_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_D_vpeq_i_pD");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_vmeq_c_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_vmeq_c_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_vmeq_c_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_vmeq_c_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_vmeq_C_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_vmeq_C_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_vmeq_C_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_vmeq_C_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_vmeq_pC_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_vmeq_pC_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_vmeq_pC_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_vmeq_pC_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_vmeq_Ca_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_vmeq_Ca_times_D");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_vmeq_Ca_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_vmeq_Ca_times_pD");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_vmeq_pCa_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_vmeq_pCa_times_D");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_vmeq_pCa_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_vmeq_pCa_times_pD");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_vmeq_R_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_vmeq_R_times_D");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_vmeq_R_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_vmeq_R_times_pD");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_vmeq_pR_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_vmeq_pR_times_D");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_vmeq_pR_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_vmeq_pR_times_pD");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_vmeq_conj_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_D_vmeq_conj_D");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_vmeq_conj_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_D_vmeq_conj_pD");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_vmeq_i_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_D_vmeq_i_D");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_vmeq_i_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_D_vmeq_i_pD");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_veqm_c_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_veqm_c_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_veqm_c_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_veqm_c_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_veqm_C_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_veqm_C_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_veqm_C_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_veqm_C_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_veqm_pC_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_veqm_pC_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_veqm_pC_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_veqm_pC_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_veqm_Ca_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_veqm_Ca_times_D");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_veqm_Ca_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_veqm_Ca_times_pD");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_veqm_pCa_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_veqm_pCa_times_D");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_veqm_pCa_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_veqm_pCa_times_pD");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_veqm_R_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_veqm_R_times_D");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_veqm_R_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_veqm_R_times_pD");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_veqm_pR_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_veqm_pR_times_D");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_veqm_pR_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_veqm_pR_times_pD");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_veqm_conj_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_D_veqm_conj_D");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_veqm_conj_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_D_veqm_conj_pD");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_veqm_i_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, int n) {
  QLAB_TRACE("QLA_D2_D_veqm_i_D");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_veqm_i_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, int n) {
  QLAB_TRACE("QLA_D2_D_veqm_i_pD");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, nullptr, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_veq_D_plus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_D_plus_D");
  qlab::api_ew_n<double, qlab::EW_PLUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_r_times_D_plus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, QLA_D2_DiracFermion *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D2_D_veq_r_times_D_plus_D");
  qlab::api_ew_n<double, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_c_times_D_plus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, QLA_D2_DiracFermion *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D2_D_veq_c_times_D_plus_D");
  qlab::api_ew_n<double, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_D_minus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_D_minus_D");
  qlab::api_ew_n<double, qlab::EW_MINUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_r_times_D_minus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, QLA_D2_DiracFermion *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D2_D_veq_r_times_D_minus_D");
  qlab::api_ew_n<double, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_c_times_D_minus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, QLA_D2_DiracFermion *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D2_D_veq_c_times_D_minus_D");
  qlab::api_ew_n<double, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_D_plus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_D_plus_pD");
  qlab::api_ew_n<double, qlab::EW_PLUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_r_times_D_plus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, QLA_D2_DiracFermion *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D2_D_veq_r_times_D_plus_pD");
  qlab::api_ew_n<double, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_c_times_D_plus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, QLA_D2_DiracFermion *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D2_D_veq_c_times_D_plus_pD");
  qlab::api_ew_n<double, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_D_minus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_D_minus_pD");
  qlab::api_ew_n<double, qlab::EW_MINUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_r_times_D_minus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, QLA_D2_DiracFermion *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D2_D_veq_r_times_D_minus_pD");
  qlab::api_ew_n<double, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_c_times_D_minus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, QLA_D2_DiracFermion *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D2_D_veq_c_times_D_minus_pD");
  qlab::api_ew_n<double, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_pD_plus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_pD_plus_D");
  qlab::api_ew_n<double, qlab::EW_PLUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_r_times_pD_plus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, QLA_D2_DiracFermion *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D2_D_veq_r_times_pD_plus_D");
  qlab::api_ew_n<double, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_c_times_pD_plus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, QLA_D2_DiracFermion *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D2_D_veq_c_times_pD_plus_D");
  qlab::api_ew_n<double, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_pD_minus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_pD_minus_D");
  qlab::api_ew_n<double, qlab::EW_MINUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_r_times_pD_minus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, QLA_D2_DiracFermion *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D2_D_veq_r_times_pD_minus_D");
  qlab::api_ew_n<double, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_c_times_pD_minus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, QLA_D2_DiracFermion *__restrict__ c, int n) {
  QLAB_TRACE("QLA_D2_D_veq_c_times_pD_minus_D");
  qlab::api_ew_n<double, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_pD_plus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_pD_plus_pD");
  qlab::api_ew_n<double, qlab::EW_PLUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_r_times_pD_plus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, QLA_D2_DiracFermion *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D2_D_veq_r_times_pD_plus_pD");
  qlab::api_ew_n<double, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_c_times_pD_plus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, QLA_D2_DiracFermion *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D2_D_veq_c_times_pD_plus_pD");
  qlab::api_ew_n<double, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_pD_minus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int n) {
  QLAB_TRACE("QLA_D2_D_veq_pD_minus_pD");
  qlab::api_ew_n<double, qlab::EW_MINUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_r_times_pD_minus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, QLA_D2_DiracFermion *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D2_D_veq_r_times_pD_minus_pD");
  qlab::api_ew_n<double, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_veq_c_times_pD_minus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, QLA_D2_DiracFermion *__restrict__ * c, int n) {
  QLAB_TRACE("QLA_D2_D_veq_c_times_pD_minus_pD");
  qlab::api_ew_n<double, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), nullptr, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_c_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_c_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_c_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_c_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_C_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_C_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_C_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_C_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_pC_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_pC_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_pC_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_pC_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_Ca_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_Ca_times_D");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_Ca_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_Ca_times_pD");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_pCa_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_pCa_times_D");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_pCa_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_pCa_times_pD");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_R_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_R_times_D");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_R_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_R_times_pD");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_pR_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_pR_times_D");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_pR_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_pR_times_pD");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_conj_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_conj_D");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_conj_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_conj_pD");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_i_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_i_D");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_i_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_i_pD");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xpeq_c_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xpeq_c_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_xpeq_c_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xpeq_c_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_xpeq_C_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xpeq_C_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_xpeq_C_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xpeq_C_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_xpeq_pC_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xpeq_pC_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_xpeq_pC_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xpeq_pC_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_xpeq_Ca_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xpeq_Ca_times_D");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_xpeq_Ca_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xpeq_Ca_times_pD");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_xpeq_pCa_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xpeq_pCa_times_D");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_xpeq_pCa_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xpeq_pCa_times_pD");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_xpeq_R_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xpeq_R_times_D");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_xpeq_R_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xpeq_R_times_pD");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_xpeq_pR_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xpeq_pR_times_D");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_xpeq_pR_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xpeq_pR_times_pD");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_xpeq_conj_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xpeq_conj_D");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_xpeq_conj_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xpeq_conj_pD");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_xpeq_i_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xpeq_i_D");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_xpeq_i_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xpeq_i_pD");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::PEQ);
}

QLAB_EXPORT void QLA_D2_D_xmeq_c_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xmeq_c_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_xmeq_c_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xmeq_c_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_xmeq_C_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xmeq_C_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_xmeq_C_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xmeq_C_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_xmeq_pC_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xmeq_pC_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_xmeq_pC_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xmeq_pC_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_xmeq_Ca_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xmeq_Ca_times_D");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_xmeq_Ca_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xmeq_Ca_times_pD");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_xmeq_pCa_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xmeq_pCa_times_D");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_xmeq_pCa_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xmeq_pCa_times_pD");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_xmeq_R_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xmeq_R_times_D");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_xmeq_R_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xmeq_R_times_pD");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_xmeq_pR_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xmeq_pR_times_D");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_xmeq_pR_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xmeq_pR_times_pD");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_xmeq_conj_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xmeq_conj_D");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_xmeq_conj_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xmeq_conj_pD");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_xmeq_i_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xmeq_i_D");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_xmeq_i_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xmeq_i_pD");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::MEQ);
}

QLAB_EXPORT void QLA_D2_D_xeqm_c_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeqm_c_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_xeqm_c_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeqm_c_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_CONST, false>("D2_ew_ctimes", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_xeqm_C_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeqm_C_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_xeqm_C_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeqm_C_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_xeqm_pC_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeqm_pC_times_D");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_xeqm_pC_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeqm_pC_times_pD");
  qlab::api_ew_n<double, qlab::EW_CT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_xeqm_Ca_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeqm_Ca_times_D");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_xeqm_Ca_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeqm_Ca_times_pD");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_xeqm_pCa_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeqm_pCa_times_D");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_xeqm_pCa_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeqm_pCa_times_pD");
  qlab::api_ew_n<double, qlab::EW_CAT, qlab::SC_FIELD, false>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_xeqm_R_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeqm_R_times_D");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_xeqm_R_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeqm_R_times_pD");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_xeqm_pR_times_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeqm_pR_times_D");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_xeqm_pR_times_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeqm_pR_times_pD");
  qlab::api_ew_n<double, qlab::EW_RT, qlab::SC_FIELD, true>("D2_ew_field", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_xeqm_conj_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeqm_conj_D");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_xeqm_conj_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeqm_conj_pD");
  qlab::api_ew_n<double, qlab::EW_CONJ, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_xeqm_i_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeqm_i_D");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_xeqm_i_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeqm_i_pD");
  qlab::api_ew_n<double, qlab::EW_I, qlab::SC_NONE, false>("D2_ew_unary", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::Opnd{}, index, n, qlab::EQM);
}

QLAB_EXPORT void QLA_D2_D_xeq_D_plus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_D_plus_D");
  qlab::api_ew_n<double, qlab::EW_PLUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_r_times_D_plus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, QLA_D2_DiracFermion *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_r_times_D_plus_D");
  qlab::api_ew_n<double, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_c_times_D_plus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, QLA_D2_DiracFermion *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_c_times_D_plus_D");
  qlab::api_ew_n<double, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_D_minus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_D_minus_D");
  qlab::api_ew_n<double, qlab::EW_MINUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_r_times_D_minus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, QLA_D2_DiracFermion *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_r_times_D_minus_D");
  qlab::api_ew_n<double, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_c_times_D_minus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, QLA_D2_DiracFermion *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_c_times_D_minus_D");
  qlab::api_ew_n<double, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_D_plus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_D_plus_pD");
  qlab::api_ew_n<double, qlab::EW_PLUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_r_times_D_plus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, QLA_D2_DiracFermion *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_r_times_D_plus_pD");
  qlab::api_ew_n<double, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_c_times_D_plus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, QLA_D2_DiracFermion *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_c_times_D_plus_pD");
  qlab::api_ew_n<double, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_D_minus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_D_minus_pD");
  qlab::api_ew_n<double, qlab::EW_MINUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_contig(a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_r_times_D_minus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, QLA_D2_DiracFermion *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_r_times_D_minus_pD");
  qlab::api_ew_n<double, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_c_times_D_minus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ b, QLA_D2_DiracFermion *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_c_times_D_minus_pD");
  qlab::api_ew_n<double, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_contig(b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_pD_plus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_pD_plus_D");
  qlab::api_ew_n<double, qlab::EW_PLUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_r_times_pD_plus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, QLA_D2_DiracFermion *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_r_times_pD_plus_D");
  qlab::api_ew_n<double, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_c_times_pD_plus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, QLA_D2_DiracFermion *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_c_times_pD_plus_D");
  qlab::api_ew_n<double, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_pD_minus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_pD_minus_D");
  qlab::api_ew_n<double, qlab::EW_MINUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_contig(b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_r_times_pD_minus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, QLA_D2_DiracFermion *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_r_times_pD_minus_D");
  qlab::api_ew_n<double, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_c_times_pD_minus_D(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, QLA_D2_DiracFermion *__restrict__ c, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_c_times_pD_minus_D");
  qlab::api_ew_n<double, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_contig(c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_pD_plus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_pD_plus_pD");
  qlab::api_ew_n<double, qlab::EW_PLUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_r_times_pD_plus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, QLA_D2_DiracFermion *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_r_times_pD_plus_pD");
  qlab::api_ew_n<double, qlab::EW_RT_PLUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_c_times_pD_plus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, QLA_D2_DiracFermion *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_c_times_pD_plus_pD");
  qlab::api_ew_n<double, qlab::EW_CT_PLUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_pD_minus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D2_DiracFermion *__restrict__ * a, QLA_D2_DiracFermion *__restrict__ * b, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_pD_minus_pD");
  qlab::api_ew_n<double, qlab::EW_MINUS, qlab::SC_NONE, false>("D2_ew_sum", 2, 4 * 2, qlab::PERM_ID, r, nullptr, qlab::Opnd{}, qlab::op_ptr((const void* const*)a), qlab::op_ptr((const void* const*)b), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_r_times_pD_minus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Real *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, QLA_D2_DiracFermion *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_r_times_pD_minus_pD");
  qlab::api_ew_n<double, qlab::EW_RT_MINUS, qlab::SC_CONST, true>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

QLAB_EXPORT void QLA_D2_D_xeq_c_times_pD_minus_pD(QLA_D2_DiracFermion *__restrict__ r, QLA_D_Complex *__restrict__ a, QLA_D2_DiracFermion *__restrict__ * b, QLA_D2_DiracFermion *__restrict__ * c, int * index, int n) {
  QLAB_TRACE("QLA_D2_D_xeq_c_times_pD_minus_pD");
  qlab::api_ew_n<double, qlab::EW_CT_MINUS, qlab::SC_CONST, false>("D2_ew_axpby", 2, 4 * 2, qlab::PERM_ID, r, a, qlab::Opnd{}, qlab::op_ptr((const void* const*)b), qlab::op_ptr((const void* const*)c), index, n, qlab::EQ);
}

}  // extern "C"
